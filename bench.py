#!/usr/bin/env python
"""Benchmark of the Dirac-operator hot path on B200.

One step = one application of the FP64 O(a)-improved Wilson-Dirac operator
Dw_dble (modules/dirac/Dw_dble.c:1377 in the reference) to a 32^3x64 lattice
(V = 2,097,152 sites; links exp(0.3 X), m0 = -0.05, csw = 1.7, bs = 4^4),
the single-operator bandwidth workload.  The metric is the algorithmic HBM
throughput, 1536 bytes per site (spinor in 192 + out 192 + 4 links 576 + SW
576), in GB/s; every application moves 3.2 GB, far more than the 126 MB L2,
so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value   : device-resident fields, K back-to-back launches timed with CUDA
          events on the library's stream, max over ranks.
e2e     : the drop-in C entry point Dw_dble(mu, s, r) on page-locked host
          arrays in the reference layout (host->device copy, layout
          conversion, operator, conversion back, device->host copy).
Extra keys report the FP32 operator and the plain GPU SAP+GCR solve
(seconds per right-hand side to FP64 relative residual 1e-10).

With N GPUs (torchrun) the ranks hold consecutive 32^3x64 slabs along x0
of one (64 N) x 32^3 lattice (the reference's NPROC0 = N process grid, weak
scaling): every application packs the half-spinor x0-faces, exchanges them
with the neighbour ranks (NCCL point-to-point, or through the host with
--dd-transport host) and then runs the operator; the timings are maxed over
the ranks.  --impl reference times the reference's own CPU Dw_dble (built
from its sources, OpenMP on the host cores) on one slab, on rank 0.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "openqcd-2.4.2_b200"))

import numpy as np  # noqa: E402

LATTICE = (64, 32, 32, 32)
BS = (4, 4, 4, 4)
EPS, M0, CSW, MU = 0.3, -0.05, 1.7, 0.0
BYTES_PER_SITE = {64: 1536, 32: 768}
WORKLOAD = "Dw_dble on 32^3x64 (links exp(0.3 X), m0=-0.05, csw=1.7, periodic gauge / antiperiodic fermion bc)"


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "20"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        # nvidia-smi needs a moment before its first sample: wait for it, so
        # that a short timed region started after this falls between samples
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 3.0:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.1)      # one more sample after the timed region
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[3 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


class Dist:
    """backend "nccl" (one GPU per rank) or "gloo" (host transport of the
    faces: ranks may share a GPU, and the CPU tests of the rank logic)"""

    def __init__(self, backend="nccl"):
        self.rank = env_int("RANK", 0)
        self.world = env_int("WORLD_SIZE", 1)
        self.local = env_int("LOCAL_RANK", 0)
        self.device = self.local
        self.pg = None
        self.cuda = False
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            has_gpu = torch.cuda.is_available()
            self.cuda = has_gpu and backend == "nccl"
            if has_gpu:
                self.device = self.local % torch.cuda.device_count()
                torch.cuda.set_device(self.device)
            # a short timeout: ranks waiting for a failed one end with an error
            dist.init_process_group("nccl" if self.cuda else "gloo", timeout=datetime.timedelta(seconds=300))
            self.torch, self.dist = torch, dist
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, x):
        if not self.pg:
            return x
        t = self.torch.tensor([float(x)], device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


FIELD_SEED, SOURCE_SEED = 20251203, 7


def expiq(Q):
    """exp(iQ) for traceless Hermitian 3x3 matrices Q[..., 3, 3], by the
    Cayley-Hamilton closed form of Morningstar and Peardon (Phys. Rev. D 69
    (2004) 054501, eqs. 19-34): exp(iQ) = f0 + f1 Q + f2 Q^2 with the f_j from
    the invariants c0 = det Q, c1 = tr Q^2 / 2; c0 < 0 through
    f_j(-c0) = (-1)^j conj(f_j(c0))."""
    Q2 = Q @ Q
    c1 = 0.5 * np.einsum("...ii->...", Q2).real
    c0 = np.einsum("...ij,...ji->...", Q, Q2).real / 3.0
    neg = c0 < 0
    c0 = np.abs(c0)
    c1s = np.maximum(c1, 1e-300)
    c0max = 2.0 * (c1s / 3.0) ** 1.5
    theta = np.arccos(np.clip(c0 / c0max, -1.0, 1.0))
    u = np.sqrt(c1s / 3.0) * np.cos(theta / 3.0)
    w = np.sqrt(c1s) * np.sin(theta / 3.0)
    w2 = w * w
    small = np.abs(w) < 0.05
    xi0 = np.where(small, 1.0 - w2 / 6.0 * (1.0 - w2 / 20.0 * (1.0 - w2 / 42.0)),
                   np.sin(w) / np.where(small, 1.0, w))
    u2 = u * u
    e2iu = np.exp(2j * u)
    emiu = np.exp(-1j * u)
    cw = np.cos(w)
    h0 = (u2 - w2) * e2iu + emiu * (8.0 * u2 * cw + 2j * u * (3.0 * u2 + w2) * xi0)
    h1 = 2.0 * u * e2iu - emiu * (2.0 * u * cw - 1j * (3.0 * u2 - w2) * xi0)
    h2 = e2iu - emiu * (cw + 3j * u * xi0)
    den = 9.0 * u2 - w2
    f0, f1, f2 = h0 / den, h1 / den, h2 / den
    f0 = np.where(neg, np.conj(f0), f0)
    f1 = np.where(neg, -np.conj(f1), f1)
    f2 = np.where(neg, np.conj(f2), f2)
    U = f1[..., None, None] * Q + f2[..., None, None] * Q2
    for i in range(3):
        U[..., i, i] += f0
    return U


def synthetic_links(L, eps, seed, planes=None):
    """U(x, mu) = exp(i eps H), H = sum_a c_a T_a with c_a ~ N(0, 1) (a
    Gaussian traceless Hermitian matrix, unit variance per su(3) generator,
    T_a the Gell-Mann matrices / 2), for every site x of the time planes
    `planes` (default all) of the lattice L (lexicographic, x3 fastest) and
    every direction mu; the time links at x0 = L0 - 1 carry the factor -1
    of the antiperiodic quark boundary (bc type 3, as set_ud_phase leaves
    the field).  Every time plane has its own random stream (seed, x0), so a
    rank can make its slab of a large lattice alone.  Returns complex128
    [len(planes) * L1 L2 L3, 4, 3, 3].  Built in numpy so that both bench
    arms run on the same field."""
    planes = list(range(L[0])) if planes is None else list(planes)
    F = int(np.prod(L[1:]))
    U = np.empty((len(planes), F, 4, 3, 3), dtype=np.complex128)
    for k, x0 in enumerate(planes):
        c = np.random.default_rng([seed, x0]).standard_normal((8, F, 4)) * (0.5 * eps)
        H = np.empty((F, 4, 3, 3), dtype=np.complex128)
        d8 = c[7] / np.sqrt(3.0)
        H[..., 0, 0] = c[2] + d8
        H[..., 1, 1] = -c[2] + d8
        H[..., 2, 2] = -2.0 * d8
        H[..., 0, 1] = c[0] - 1j * c[1]
        H[..., 0, 2] = c[3] - 1j * c[4]
        H[..., 1, 2] = c[5] - 1j * c[6]
        H[..., 1, 0] = np.conj(H[..., 0, 1])
        H[..., 2, 0] = np.conj(H[..., 0, 2])
        H[..., 2, 1] = np.conj(H[..., 1, 2])
        U[k] = expiq(H)
        if x0 == L[0] - 1:
            U[k, :, 0] *= -1.0
    return U.reshape(-1, 4, 3, 3)


def synthetic_source(L, seed, planes=None):
    """Gaussian spinor field, unit variance per real component, [V, 24]
    (lexicographic sites of the time planes `planes`, one random stream
    per plane)."""
    planes = list(range(L[0])) if planes is None else list(planes)
    F = int(np.prod(L[1:]))
    return np.concatenate([np.random.default_rng([seed, x0]).standard_normal((F, 24)) for x0 in planes])


def slab_links_storage(Lg, x0a, L0, eps, seed, ipt):
    """The reference's gauge-field array, storage order ipt[] (ipt[lex] =
    storage index, even sites first), of the slab x0a <= x0 < x0a + L0 of the
    global lattice Lg: U(x, mu) at slot 8 (ix - V/2) + 2 mu of the odd site x
    with index ix, U(x - mu, mu) at slot 8 (ix - V/2) + 2 mu + 1
    (main/README.global); for the first plane's odd sites U(x - 0, 0) is a
    link of the plane below the slab, as openQCD's local fields hold it."""
    Ll = (L0,) + tuple(Lg[1:])
    V = int(np.prod(Ll))
    below = synthetic_links(Lg, eps, seed, [(x0a - 1) % Lg[0]])          # the plane below
    U = synthetic_links(Lg, eps, seed, range(x0a, x0a + L0))
    x = np.indices(Ll).reshape(4, -1)
    odd = np.nonzero(x.sum(axis=0) & 1)[0]
    base = 8 * (ipt[odd].astype(np.int64) - V // 2)
    out = np.empty((4 * V, 3, 3), dtype=np.complex128)
    xo = x[:, odd]
    for mu in range(4):
        out[base + 2 * mu] = U[odd, mu]
        y = xo.copy()
        y[mu] = (y[mu] - 1) % Ll[mu]
        lex_m = np.ravel_multi_index(tuple(y), Ll)
        bw = U[lex_m, mu]
        if mu == 0:
            first = xo[0] == 0
            bw[first] = below[np.ravel_multi_index(tuple(xo[1:, first]), Lg[1:]), 0]
        out[base + 2 * mu + 1] = bw
    return out.view(np.float64).reshape(-1)


def spinor_storage(s_lex, ipt):
    out = np.empty_like(s_lex)
    out[ipt] = s_lex
    return out.reshape(-1)


def max_site_err(a_store, b_store, ipt_a, ipt_b):
    """max over sites of |a(x) - b(x)| / |b(x)| for two spinor fields in
    the storage orders ipt_a, ipt_b"""
    a = np.asarray(a_store, dtype=np.float64).reshape(-1, 24)[ipt_a]
    b = np.asarray(b_store, dtype=np.float64).reshape(-1, 24)[ipt_b]
    return float((np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max())


DATA = "synthetic: links exp(i 0.3 H), H Gaussian traceless Hermitian, and a Gaussian source, made in numpy"


def bench_config(ngpus):
    """the workload description both arms print: with N GPUs, N slabs of
    32^3x64 along x0 (global lattice (64 N) x 32^3, weak scaling)"""
    return {"workload": WORKLOAD, "lattice": list(LATTICE), "block": list(BS), "global_batch": 1,
            "parallelism": "single" if ngpus <= 1 else "x0-slabs%d (global %dx%dx%dx%d)" % (
                ngpus, ngpus * LATTICE[0], LATTICE[1], LATTICE[2], LATTICE[3]),
            "field": "numpy links exp(i 0.3 H), H Gaussian traceless Hermitian (seed %d), Gaussian source (seed %d)"
                     % (FIELD_SEED, SOURCE_SEED),
            "l2": "inputs larger than L2 (3.2 GB per application), no flush"}


def ref_lattice_threads():
    """Thread-local lattice for the reference build: as many OpenMP threads as
    host cores allow (NTHREAD = V / V_TRD, a power of two up to 64)."""
    n = os.cpu_count() or 8
    for nt, T in ((64, (16, 16, 16, 8)), (32, (16, 16, 16, 16)), (16, (32, 16, 16, 16)), (8, (32, 16, 16, 32))):
        if nt <= n:
            return nt, T
    return 8, (32, 16, 16, 32)


def reference_lib(L):
    """The reference oracle library for the bench lattice (CPU baseline only)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reflib
    nt, T = ref_lattice_threads()
    while True:
        if reflib.available(L, T) or reflib.ensure_built(L, T):
            return reflib.RefLib(L, T), nt
        # fall back to fewer threads if that build is not present
        if nt == 8:
            return None, 0
        nt //= 2
        T = {32: (16, 16, 16, 16), 16: (32, 16, 16, 16), 8: (32, 16, 16, 32)}[nt]


def bench_inputs(ipt, nproc=1, rank=0):
    """the bench's gauge field and source in storage order ipt[]: the slab of
    rank `rank` of nproc ranks along x0 (each holding a 32^3x64 slab of the
    global (64 nproc) x 32^3 lattice); nproc = 1 is the 32^3x64 lattice"""
    L0 = LATTICE[0]
    Lg = (nproc * L0,) + tuple(LATTICE[1:])
    ud = slab_links_storage(Lg, rank * L0, L0, EPS, FIELD_SEED, ipt)
    s = spinor_storage(synthetic_source(Lg, SOURCE_SEED, range(rank * L0, (rank + 1) * L0)), ipt)
    return ud, s


def reference_on_bench_field(ref):
    """load the bench's field into the reference library (its own storage
    order) and build its SW term; returns (ipt, source)"""
    ref.init(bc=3, seed=4321, csw=CSW, m0=M0, eoflg=0)
    ipt = ref.ipt()
    ud, s = bench_inputs(ipt)
    ref.set_ud(ud)
    del ud
    ref.sw_term(0)
    return ipt, s


def cpu_reference_timing(seconds=12.0, check=None):
    """Time the reference's Dw_dble (its own CPU code, OpenMP) on the bench
    field and source.  check = (device-order ipt, device result of Dw_dble
    on that source): the result is compared site by site.  Returns the
    cpu_baseline object."""
    ref, nt = reference_lib(LATTICE)
    if ref is None:
        return None
    ipt, s = reference_on_bench_field(ref)
    t1, r = ref.time_dirac_src(MU, s, 1)
    n = max(2, int(seconds / max(t1, 1e-3)))
    t, r = ref.time_dirac_src(MU, s, n)
    gbs = BYTES_PER_SITE[64] * ref.vol * n / t / 1e9
    out = {"value": gbs, "unit": "GB/s", "cores": nt, "kind": "reference",
           "sample": "%d applications of the reference Dw_dble (AVX/FMA3 build, NPROC=1, NTHREAD=%d) on the bench's "
                     "32^3x64 field and source, %.1f s" % (n, nt, t)}
    if check is not None:
        # the device's Dw_dble and Dw results on the same source, against
        # the reference's (bars 1e-13 and 2e-6 per site)
        ipt_dev, r_dev, r32_dev = check
        out["max_site_rel_err_vs_device"] = max_site_err(r_dev, r, ipt_dev, ipt)
        if r32_dev is not None:
            r32 = ref.dirac(0, MU, s.astype(np.float32))
            out["max_site_rel_err_vs_device_f32"] = max_site_err(r32_dev, r32, ipt_dev, ipt)
    return out


def run_reference(args, d):
    if d.rank != 0:
        return 0
    ref, nt = reference_lib(LATTICE)
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle library for 32^3x64 is not built"}))
        return 0
    ipt, s = reference_on_bench_field(ref)
    ref.time_dirac_src(MU, s, max(1, args.warmup))
    times = [ref.time_dirac_src(MU, s, 1)[0] for _ in range(args.steps)]
    tot = sum(times)
    gbs = BYTES_PER_SITE[64] * ref.vol * args.steps / tot / 1e9
    out = {
        "impl": "reference", "metric": "Dw_dble GB/s", "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": DATA, "config": bench_config(args.gpus),
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": nt, "kind": "reference",
                         "sample": "%d single applications of the reference Dw_dble (AVX/FMA3 build, NPROC=1, "
                                   "NTHREAD=%d) on the bench's field and source" % (args.steps, nt)},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--lattice", default=None, help="L0,L1,L2,L3 (profiling runs)")
    ap.add_argument("--dd-transport", default="nccl", choices=["nccl", "host"],
                    help="N > 1: faces between the GPUs with NCCL, or through the host with gloo (ranks sharing "
                         "a GPU)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solver", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile-solver", action="store_true",
                    help="run only the 48^3x96 solver comparison, with profiler collection around the chosen solve")
    ap.add_argument("--solver-lattice", default=None, help="L0,L1,L2,L3 for --profile-solver (smaller cases)")
    ap.add_argument("--sustained", type=int, default=0,
                    help="run only Dw_dble n times back to back, its time per launch binned by the sampled SM clock")
    ap.add_argument("--scan-block-orders", action="store_true",
                    help="run only Dw_dble under each block traversal order (timings; the first 10 launches "
                         "are the ones an ncu traffic capture takes)")
    ap.add_argument("--profile-setup", action="store_true",
                    help="run only the deflation subspace generation of the solver workload, with profiler "
                         "collection around it, and print its phase times")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    d = Dist("gloo" if args.dd_transport == "host" else "nccl")
    try:
        if args.impl == "reference":
            return run_reference(args, d)
        if args.sustained:
            import openqcd_b200 as qb
            qb.set_device(d.local)
            print(json.dumps(sustained_dw(qb, args.sustained)))
            return 0
        if args.scan_block_orders:
            import openqcd_b200 as qb
            qb.set_device(d.local)
            print(json.dumps(scan_block_orders(qb)))
            return 0
        if args.profile_setup:
            import openqcd_b200 as qb
            qb.set_device(d.local)
            L = tuple(int(x) for x in args.solver_lattice.split(",")) if args.solver_lattice else None
            print(json.dumps(setup_profile(qb, lattice=L)))
            return 0
        if args.profile_solver:
            import openqcd_b200 as qb
            qb.set_device(d.local)
            L = tuple(int(x) for x in args.solver_lattice.split(",")) if args.solver_lattice else None
            print(json.dumps(solver_c3(qb, profile=True, lattice=L)))
            return 0
        return run_b200(args, d)
    finally:
        d.close()


SOLVER_L = (96, 48, 48, 48)
SOLVER_BS = (6, 6, 6, 6)


def true_residual(qb, mu, eta, psi):
    """|eta - Dw psi| / |eta| in FP64 on the device."""
    chk = qb.DevField(64)
    qb.dev_dirac("Dw", mu, psi, chk)
    d = chk.to_ref(qb.lib().b200_volume()) - eta.to_ref(qb.lib().b200_volume())
    n = np.linalg.norm(d) / np.sqrt(eta.norm2())
    chk.free()
    return float(n)


def solver_c3(qb, profile=False, lattice=None):
    """The mixed-precision deflated solve on 48^3x96 (links exp(0.3 X),
    m0 = -0.05, csw = 1.7, bs = 6^4, Ns = 28, Gaussian sources, FP64
    residual 1e-10): the plain GPU sap_gcr (one right-hand side, FP32 SAP
    with nkv = 16, ncy = 5) against the chosen solver (deflated SAP+GCR on
    four right-hand sides at once, nkv = 8, nmr = 3, ncy = 2).  Seconds per
    right-hand side of the solves; the subspace generation is reported
    apart (it is done once per gauge field)."""
    L, BSx, NS = (lattice or SOLVER_L), SOLVER_BS, 28
    qb.geometry(L, BSx, qb.even_first_ipt(L))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 20251204)
    qb.sw_term()
    out = {"workload": "48^3x96, links exp(0.3 X), m0=-0.05, csw=1.7, bs=6^4, Gaussian sources, res 1e-10",
           "data": "synthetic"}
    qb.set_sap_parms(BSx, 1, 4, 5)
    eta = qb.DevField(64).random(1.0, 9)
    psi = qb.DevField(64)
    qb.dev_sap_gcr(16, 1024, 0, 1e-10, 0.0, eta, psi)    # warm-up (and SAP autotuning)
    qb.lib().b200_sync()
    t0 = time.time()
    rho, ifail, st = qb.dev_sap_gcr(16, 1024, 0, 1e-10, 0.0, eta, psi)
    qb.lib().b200_sync()
    t_plain = time.time() - t0
    out["plain"] = {"s_per_rhs": t_plain, "iterations": st, "ifail": ifail,
                    "true_residual": true_residual(qb, 0.0, eta, psi),
                    "solver": "sap_gcr: nkv=16, isolv=1, nmr=4, ncy=5, FP32 SAP/Krylov, FP64 residual"}
    qb.release_workspace()
    qb.set_dfl_parms(BSx, NS)
    qb.set_dfl_pro_parms(24, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 + M0)), 0.0, 10, 4, 4)
    t0 = time.time()
    f, stm = qb.dfl_modes(1)
    qb.lib().b200_sync()
    t_setup = time.time() - t0
    qb.release_workspace()      # the generation's work fields
    nr = 4
    qb.set_sap_parms(BSx, 1, 3, 2)
    E = [eta] + [qb.DevField(64).random(1.0, 100 + i) for i in range(nr - 1)]
    P = [qb.DevField(64) for _ in range(nr)]
    qb.dev_gcr_batch(8, 256, 0, 1e-10, [0.0] * nr, E, P, dfl=True)      # warm-up
    qb.lib().b200_sync()
    if profile:
        qb.check(qb.lib().b200_profiler(1))
    t0 = time.time()
    rhos, ifails, sts, lst = qb.dev_gcr_batch(8, 256, 0, 1e-10, [0.0] * nr, E, P, dfl=True)
    qb.lib().b200_sync()
    t_chosen = (time.time() - t0) / nr
    if profile:
        qb.check(qb.lib().b200_profiler(0))
    out["chosen"] = {"s_per_rhs": t_chosen, "iterations": sts, "little_steps": lst, "ifail": ifails,
                     "true_residual": max(true_residual(qb, 0.0, E[i], P[i]) for i in range(nr)),
                     "setup_s": t_setup, "setup_ifail": f,
                     "solver": "dfl_sap_gcr batched over 4 right-hand sides: Ns=28 deflation (subspace by "
                               "dfl_modes, ninv=10), nkv=8, isolv=1, nmr=3, ncy=2, FP32 SAP/Krylov, FP64 "
                               "residual, multi-RHS restriction/prolongation/little solver"}
    out["speedup_per_rhs"] = t_plain / t_chosen
    # right-hand sides per gauge field after which the subspace generation
    # has paid for itself
    out["break_even_rhs"] = t_setup / (t_plain - t_chosen) if t_plain > t_chosen else None
    for fld in E + P:
        fld.free()
    psi.free()
    qb.release_workspace()
    return out


def sustained_dw(qb, n, chunk=20):
    """Dw_dble on the bench's 32^3x64 field, n launches back to back in
    chunks of `chunk` (CUDA events per chunk, wall-clock stamps around it),
    with nvidia-smi sampling the SM clock and power every 20 ms: each
    chunk's time per launch paired with the median clock sampled during it,
    then binned by clock (100 MHz bins).  For the record of how the kernel
    behaves once the power cap pulls the clock down; the bench's own timed
    region is the short burst of --steps launches."""
    import datetime
    L = LATTICE
    qb.geometry(L, BS, qb.even_first_ipt(L))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, FIELD_SEED)
    qb.sw_term()
    s = qb.DevField(64).random(1.0, SOURCE_SEED)
    r = qb.DevField(64)
    vol = qb.lib().b200_volume()
    qb.time_dirac(64, "Dw", MU, s, r, 5)
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    p = subprocess.Popen(["nvidia-smi", "-i", "0", "--query-gpu=timestamp,clocks.sm,power.draw,"
                          "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "20"],
                         stdout=f, stderr=subprocess.DEVNULL)
    time.sleep(1.0)
    chunks = []
    for _ in range(max(1, n // chunk)):
        t0 = time.time()
        ms = qb.time_dirac(64, "Dw", MU, s, r, chunk) / chunk
        chunks.append((t0, time.time(), ms))
    time.sleep(0.2)
    p.terminate()
    p.wait(timeout=5)
    f.flush()
    samples = []
    for line in open(f.name):
        parts = [x.strip() for x in line.split(",")]
        if len(parts) != 4:
            continue
        try:
            ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            samples.append((ts, float(parts[1]), float(parts[2]), parts[3].lower().startswith("active")))
        except ValueError:
            continue
    os.unlink(f.name)
    peak = peaks()[0]
    rows = []
    for t0, t1, ms in chunks:
        inside = [x for x in samples if t0 <= x[0] <= t1]
        if not inside:   # a chunk shorter than the sampling interval: the nearest sample
            inside = [min(samples, key=lambda x: abs(x[0] - 0.5 * (t0 + t1)))] if samples else []
        if inside:
            rows.append((statistics.median(x[1] for x in inside), ms, max(x[2] for x in inside),
                         any(x[3] for x in inside)))
    bins = {}
    for mhz, ms, w, cap in rows:
        b = int(mhz // 100) * 100
        bins.setdefault(b, []).append((ms, w, cap))
    out = {"lattice": list(L), "launches": len(chunks) * chunk, "chunk": chunk,
           "ms_first_chunk": chunks[0][2], "ms_last_chunk": chunks[-1][2],
           "ms_mean": statistics.mean(c[2] for c in chunks), "bins": []}
    for b in sorted(bins):
        v = bins[b]
        msm = statistics.mean(x[0] for x in v)
        out["bins"].append({"sm_mhz": [b, b + 100], "chunks": len(v), "ms_per_launch": msm,
                            "frac_of_measured": BYTES_PER_SITE[64] * vol / (msm / 1e3) / 1e9 / peak,
                            "max_power_w": max(x[1] for x in v), "sw_power_cap": any(x[2] for x in v)})
    s.free()
    r.free()
    return out


def scan_block_orders(qb):
    """Dw_dble on 32^3x64 under each block traversal order: first two
    launches per order (the launches a 10-launch ncu capture of
    dirac_staged sees), then 3 x 20 timed launches per order."""
    L = LATTICE
    qb.geometry(L, BS, qb.even_first_ipt(L))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, FIELD_SEED)
    qb.sw_term()
    s = qb.DevField(64).random(1.0, SOURCE_SEED)
    r = qb.DevField(64)
    vol = qb.lib().b200_volume()
    for k in range(5):
        qb.set_block_order(k)
        qb.dev_dirac("Dw", 0.0, s, r)
        qb.dev_dirac("Dw", 0.0, s, r)
    out = {}
    for k in range(5):
        qb.set_block_order(k)
        qb.time_dirac(64, "Dw", 0.0, s, r, 5)
        ms = [qb.time_dirac(64, "Dw", 0.0, s, r, 20) / 20 for _ in range(3)]
        out[k] = {"ms": ms, "GBs": BYTES_PER_SITE[64] * vol / (min(ms) / 1e3) / 1e9}
    qb.set_block_order(0)
    return out


def setup_profile(qb, lattice=None):
    """Subspace generation of the solver workload (dfl_modes, Ns = 28, ninv =
    10, on the solver's field) with profiler collection around it: seconds
    and the phase timers of the deflation code."""
    L, BSx, NS = (lattice or SOLVER_L), SOLVER_BS, 28
    qb.geometry(L, BSx, qb.even_first_ipt(L))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 20251204)
    qb.sw_term()
    qb.set_sap_parms(BSx, 1, 4, 5)
    qb.set_dfl_parms(BSx, NS)
    qb.set_dfl_pro_parms(24, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 + M0)), 0.0, 10, 4, 4)
    qb.dfl_profile(True)
    qb.check(qb.lib().b200_profiler(1))
    t0 = time.time()
    f, st = qb.dfl_modes(1)
    qb.lib().b200_sync()
    dt = time.time() - t0
    qb.check(qb.lib().b200_profiler(0))
    return {"lattice": list(L), "dfl_modes_s": dt, "ifail": f, "status": st, "phases_s": qb.dfl_profile(False)}


def batched_c4(qb):
    """The batched workload on 32^3x64 (links exp(0.3 X), m0 = -0.05,
    csw = 1.7): 12 spin-colour point sources at a seeded site times the
    twisted masses mu = 0, 0.005, 0.02, 0.08, 48 systems, to FP64 residual
    1e-10, in two batches of 24 systems of the deflated solver, two masses
    per batch (Ns = 28 subspace generated once, one little operator per
    mass; nkv = 8, nmr = 4, ncy = 2); systems leave their batch as they
    converge.  The SAP block
    (also the DFL block) is picked by the block-shape autotuner, each
    candidate scored by the deflated solver's convergence per second on its
    own subspace; the RHS tile of the restriction/prolongation by the
    RHS-tile autotuner.  The plain sap_gcr (4^4 blocks, nmr = 4, ncy = 5) on the
    first source of each mass is timed beside it."""
    L = LATTICE
    ipt = qb.even_first_ipt(L)
    qb.geometry(L, BS, ipt)
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 20251205)
    qb.sw_term()
    rng = np.random.default_rng(12345)
    x0 = [int(rng.integers(0, L[m])) for m in range(4)]
    mus = [0.0, 0.005, 0.02, 0.08]
    out = {"workload": "32^3x64, 12 point sources at %s x mu in %s = 48 systems, res 1e-10" % (x0, mus),
           "data": "synthetic"}

    def sources():
        return [qb.DevField(64).point(x0, a, b) for a in range(4) for b in range(3)]

    qb.set_sap_parms(BS, 1, 4, 5)
    srcs = sources()
    psi = qb.DevField(64)
    qb.dev_sap_gcr(16, 1024, 0, 1e-10, 0.0, srcs[0], psi)
    plain = []
    for mu in mus:
        qb.lib().b200_sync()
        t0 = time.time()
        rho, ifail, st = qb.dev_sap_gcr(16, 1024, 0, 1e-10, mu, srcs[0], psi)
        qb.lib().b200_sync()
        plain.append({"mu": mu, "s": time.time() - t0, "iterations": st})
    out["plain_first_source"] = plain
    for f in srcs + [psi]:
        f.free()
    qb.release_workspace()
    # block shape (SAP and DFL block) for the chosen solver: every candidate
    # with its own 28-mode subspace, scored by the deflated solver's residual
    # reduction per second (SAP nmr = 4, ncy = 2)
    cands = [(4, 4, 4, 4), (8, 4, 4, 4), (4, 4, 4, 8), (4, 4, 8, 8)]
    qb.set_dfl_pro_parms(24, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 + M0)), 0.0, 10, 4, 4)
    qb.set_sap_parms(BS, 1, 4, 2)
    t0 = time.time()
    bs, scores = qb.tune_block_shape(cands, nsteps=6, mu=0.0, Ns=28)
    out["block_shape"] = {"candidates": [list(c) for c in cands], "score_ln_reduction_per_s": scores,
                          "chosen": list(bs), "s": time.time() - t0,
                          "objective": "deflated SAP+GCR steps, a 28-mode subspace per candidate"}
    qb.set_dfl_parms(bs, 28)
    qb.set_sap_parms(bs, 1, 4, 5)
    t0 = time.time()
    qb.dfl_modes(2)
    qb.lib().b200_sync()
    setup = time.time() - t0
    qb.set_sap_parms(bs, 1, 4, 2)
    srcs = sources()
    # two batches of 24 systems, two masses each (48 systems at once would
    # need 48 x (2 nkv + 2) FP32 Krylov fields of 201 MB, more than the 180 GB)
    P = [qb.DevField(64) for _ in range(24)]
    # warm-up with the shape of a timed batch (work fields of 24 systems,
    # the two-mass little operators, the captured SAP sequences)
    qb.dev_gcr_batch(8, 256, 0, 1e-10, [mus[i // 12] for i in range(24)], [srcs[i % 12] for i in range(24)], P,
                     dfl=True)
    # two timed passes over the 48 systems (a pass: both batches, each
    # timed alone); the faster pass is the figure, both are reported (a
    # batch now and then stalls for up to a second outside the solver's own
    # work, with the same iteration counts)
    worst, passes = 0.0, []
    for ps in range(2):
        tot, per_mu, batches = 0.0, [], []
        for pair in ((0, 1), (2, 3)):
            E = [srcs[i % 12] for i in range(24)]
            M = [mus[pair[i // 12]] for i in range(24)]
            qb.lib().b200_sync()
            t0 = time.time()
            rho, ifail, st, lst = qb.dev_gcr_batch(8, 256, 0, 1e-10, M, E, P, dfl=True)
            qb.lib().b200_sync()
            dt = time.time() - t0
            tot += dt
            batches.append({"mu": [mus[pair[0]], mus[pair[1]]], "s": dt})
            worst = max(worst, max(true_residual(qb, M[i], E[i], P[i]) for i in range(24)))
            for k in range(2):
                per_mu.append({"mu": mus[pair[k]], "iterations": st[12 * k:12 * k + 12],
                               "little_steps": lst[12 * k:12 * k + 12], "ifail": ifail[12 * k:12 * k + 12]})
        passes.append((tot, batches, per_mu))
    tot, batches, per_mu = min(passes, key=lambda x: x[0])
    out["chosen"] = {"systems": 48, "s_total": tot, "solves_per_s": 48 / tot, "s_per_rhs": tot / 48,
                     "timing": "the faster of two passes over the 48 systems",
                     "passes_s": [x[0] for x in passes], "passes_batches": [x[1] for x in passes],
                     "batches": batches, "per_mass": per_mu, "setup_s": setup, "true_residual_max": worst,
                     "block": list(bs),
                     "solver": "deflated SAP+GCR, two batches of 24 (two masses each, one little operator per "
                               "mass), Ns=28, nkv=8, nmr=4, ncy=2, autotuned block shape and RHS tile"}
    out["plain_s_per_rhs_mean"] = sum(p["s"] for p in plain) / len(plain)
    out["speedup_per_rhs"] = out["plain_s_per_rhs_mean"] / out["chosen"]["s_per_rhs"]
    gain = out["plain_s_per_rhs_mean"] - out["chosen"]["s_per_rhs"]
    # right-hand sides per gauge field that pay for the subspace (and, once
    # per lattice and parameter set, for the block-shape tuning as well)
    out["break_even_rhs"] = setup / gain if gain > 0 else None
    out["break_even_rhs_with_tuning"] = (setup + out["block_shape"]["s"]) / gain if gain > 0 else None
    out["rhs_tiles"] = qb.rhs_tiles()
    for f in srcs + P:
        f.free()
    qb.release_workspace()
    return out


def learned_c5(qb):
    """The learned preconditioner: a gauge-equivariant parallel-transport
    network (4-8-8-4 colour-triplet channels, FP16 weights at inference)
    trained on the device on 2048 (source, solution) pairs from the plain
    solver on a 16^4 field (links exp(0.3 X), m0 = -0.05, csw = 1.7), and a
    second one trained on 512 (residual, SAP-error) pairs (the error
    Dw^-1 r - M_sap r that five SAP cycles leave), then used as the
    flexible-GCR preconditioner on a 32^3x64 field and on a 48^3x96 field
    (6^4 SAP blocks): GCR steps and seconds to FP64 residual 1e-10 with no
    preconditioner (32^3x64 only), the network (SAP when it stalls), SAP,
    the network followed by SAP, and SAP plus the SAP-error network."""
    out = {"data": "synthetic"}
    L16 = (16, 16, 16, 16)
    qb.geometry(L16, BS, qb.even_first_ipt(L16))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 777)
    qb.sw_term()
    qb.set_sap_parms(BS, 1, 4, 5)
    n = 2048
    rs = [qb.DevField(32) for _ in range(n)]
    es = [qb.DevField(32) for _ in range(n)]
    t0 = time.time()
    qb.net_make_pairs(rs, es, 0.0, 1e-6, seed=3)
    out["pairs"] = {"n": n, "lattice": list(L16), "s": time.time() - t0}
    qb.net_init(1, 0.25)
    t0 = time.time()
    hist = qb.net_train(rs, es, 1200, 8, 3e-3, seed=9)
    qb.lib().b200_sync()
    out["training"] = {"steps": 1200, "batch": 8, "lr": 3e-3, "s": time.time() - t0,
                       "loss_first": float(hist[:10].mean()), "loss_last": float(hist[-50:].mean())}
    w = qb.net_get_weights()
    # a second network, trained on (residual, SAP-error) pairs, added to SAP
    # (M = M_sap + N): it learns what SAP leaves rather than the whole inverse
    nsap = 512
    t0 = time.time()
    qb.net_make_sap_pairs(rs[:nsap], es[:nsap], 0.0, 1e-6, seed=4)
    out["sap_error_pairs"] = {"n": nsap, "s": time.time() - t0}
    qb.net_init(2, 0.1)
    t0 = time.time()
    hist2 = qb.net_train(rs[:nsap], es[:nsap], 600, 8, 3e-3, seed=10)
    qb.lib().b200_sync()
    out["sap_error_training"] = {"steps": 600, "batch": 8, "lr": 3e-3, "s": time.time() - t0,
                                 "loss_first": float(hist2[:10].mean()), "loss_last": float(hist2[-50:].mean())}
    w_sap = qb.net_get_weights()
    for f in rs + es:
        f.free()
    qb.release_workspace()
    qb.geometry(LATTICE, BS, qb.even_first_ipt(LATTICE))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 20251206)
    qb.sw_term()
    qb.set_sap_parms(BS, 1, 4, 5)
    qb.net_set_weights(w)
    eta = qb.DevField(64).random(1.0, 31)
    psi = qb.DevField(64)
    res = {}
    for kind, name in ((0, "sap"), (1, "network"), (2, "network+sap"), (3, "none"), (4, "sap+error-network")):
        qb.net_set_weights(w_sap if kind == 4 else w)
        qb.set_precond(kind)
        qb.dev_sap_gcr(16, 8192, 0, 1e-10, 0.0, eta, psi) if kind != 3 else None
        qb.lib().b200_sync()
        t0 = time.time()
        rho, ifail, st = qb.dev_sap_gcr(16, 8192, 0, 1e-10, 0.0, eta, psi)
        qb.lib().b200_sync()
        res[name] = {"s": time.time() - t0, "iterations": st, "ifail": ifail,
                     "true_residual": true_residual(qb, 0.0, eta, psi)}
    qb.set_precond(0)
    out["solve_32x64"] = res
    eta.free(); psi.free()
    qb.release_workspace()
    # the same network on the 48^3x96 field of the deflated solve (6^4 blocks)
    qb.geometry(SOLVER_L, SOLVER_BS, qb.even_first_ipt(SOLVER_L))
    qb.set_parms(CSW, M0, 0)
    qb.random_ud(EPS, 20251204)
    qb.sw_term()
    qb.set_sap_parms(SOLVER_BS, 1, 4, 5)
    qb.net_set_weights(w)
    eta = qb.DevField(64).random(1.0, 9)
    psi = qb.DevField(64)
    qb.set_precond(0)
    qb.dev_sap_gcr(16, 2, 0, 1e-10, 0.0, eta, psi)      # SAP autotuning for the 6^4 blocks, untimed
    res = {}
    for kind, name in ((0, "sap"), (1, "network"), (2, "network+sap"), (4, "sap+error-network")):
        qb.net_set_weights(w_sap if kind == 4 else w)
        qb.set_precond(kind)
        qb.lib().b200_sync()
        t0 = time.time()
        rho, ifail, st = qb.dev_sap_gcr(16, 8192, 0, 1e-10, 0.0, eta, psi)
        qb.lib().b200_sync()
        res[name] = {"s": time.time() - t0, "iterations": st, "ifail": ifail,
                     "true_residual": true_residual(qb, 0.0, eta, psi)}
    qb.set_precond(0)
    out["solve_48x96"] = res
    eta.free(); psi.free()
    qb.release_workspace()
    return out


def run_b200(args, d):
    import openqcd_b200 as qb
    L = tuple(int(x) for x in args.lattice.split(",")) if args.lattice else LATTICE
    qb.set_device(d.device)
    ipt = qb.even_first_ipt(L)
    if d.world > 1:
        # the ranks hold consecutive x0-slabs of one lattice (the reference's
        # NPROC0 = N process grid), faces exchanged at every application
        dd = qb.DomainDecomposition(transport=args.dd_transport)
        dd.install()
    qb.geometry(L, BS, ipt)
    qb.set_parms(CSW, M0, 0)
    s_host = None
    if L == LATTICE:
        # the field and source the reference arm uses (both arms make them
        # in numpy from the same seeds); the SW term is built on the device
        ud, s_host = bench_inputs(ipt, d.world, d.rank)
        qb.upload_ud(ud)
        del ud
    else:
        qb.random_ud(EPS, FIELD_SEED)
    qb.sw_term()
    vol = qb.lib().b200_volume()
    s = qb.DevField(64).from_ref(s_host) if s_host is not None else qb.DevField(64).random(1.0, SOURCE_SEED)
    r = qb.DevField(64)

    clk = Clocks(d.local)      # sampling from before the warm-up to just after the timed launches
    for _ in range(args.warmup):
        qb.time_dirac(64, "Dw", MU, s, r, 1)
    d.barrier()
    qb.lib().b200_sync()
    ms = qb.time_dirac(64, "Dw", MU, s, r, args.steps)
    clocks = clk.stop()
    qb.lib().b200_sync()
    d.barrier()
    ms_max = d.max(ms)
    bytes_step = BYTES_PER_SITE[64] * vol
    value = d.world * bytes_step * args.steps / (ms_max / 1e3) / 1e9
    per_launch_ms = ms / args.steps
    peak, peak_kind = peaks()
    achieved = bytes_step / (per_launch_ms / 1e3) / 1e9

    # the result of the timed launches, for the comparison with the reference
    r_host = r.to_ref(vol) if s_host is not None else None

    extra = {}
    # FP32 operator (Dw, modules/dirac/Dw.c:973) on the same source
    s32 = qb.DevField(32).from_ref(s_host.astype(np.float32)) if s_host is not None else \
        qb.DevField(32).random(1.0, 8)
    r32 = qb.DevField(32)
    qb.time_dirac(32, "Dw", MU, s32, r32, 3)
    ms32 = qb.time_dirac(32, "Dw", MU, s32, r32, args.steps) / args.steps
    r32_host = r32.to_ref(vol) if s_host is not None else None
    # 672 algorithmic bytes per site when the links are read as 12 reals
    # (two rows, the third rebuilt), 768 with all 18
    b32 = 672 if qb.links12_active() else BYTES_PER_SITE[32]
    extra["dw_f32"] = {"ms": ms32, "GBs": b32 * vol / (ms32 / 1e3) / 1e9, "bytes_per_site": b32,
                       "frac_of_peak": b32 * vol / (ms32 / 1e3) / 1e9 / peak}
    # Dwhat_dble: 1344 algorithmic bytes per site (s_e in and r_e out, links
    # and both parities' SW matrices once); its two launches (odd sites:
    # A_oo^-1 D_oe s_e into a scratch field, even sites: the SW term minus
    # D_eo of the scratch) read every link twice, s_e twice and move the
    # scratch field out and in: 2208 bytes per site at the least
    for op, bps, moved in (("Dwhat", 1344, 2208), ):
        qb.time_dirac(64, op, MU, s, r, 3)
        m = qb.time_dirac(64, op, MU, s, r, args.steps) / args.steps
        extra["dwhat_f64"] = {"ms": m, "GBs": bps * vol / (m / 1e3) / 1e9, "bytes_per_site": bps,
                              "frac_of_peak": bps * vol / (m / 1e3) / 1e9 / peak,
                              "two_launch_bytes_per_site": moved,
                              "two_launch_frac_of_peak": moved * vol / (m / 1e3) / 1e9 / peak}
    s32.free(); r32.free()

    e2e = None
    if not args.no_e2e:
        d.barrier()
        sh = qb.HostArray(vol * 24)
        rh = qb.HostArray(vol * 24)
        qb.check(qb.lib().b200_dev_to_ref(64, s.ptr, sh.a.ctypes.data))
        qb.time_Dw_dble_host(MU, sh.a, rh.a, 2)
        n_e2e = max(3, min(args.steps, 10))
        d.barrier()
        ms_e = qb.time_Dw_dble_host(MU, sh.a, rh.a, n_e2e)
        ms_e = d.max(ms_e)
        e2e = {"value": d.world * bytes_step * n_e2e / (ms_e / 1e3) / 1e9, "unit": "GB/s",
               "h2d_bytes_per_step": vol * 192, "d2h_bytes_per_step": vol * 192,
               "ms_per_step": ms_e / n_e2e}
        sh.free(); rh.free()

    if not args.no_solver:
        qb.set_sap_parms(BS, 1, 4, 5)
        eta = qb.DevField(64).random(1.0, 9)
        psi = qb.DevField(64)
        qb.dev_sap_gcr(16, 256, 0, 1e-10, MU, eta, psi)   # warm-up
        qb.lib().b200_sync()
        t0 = time.time()
        rho, ifail, st = qb.dev_sap_gcr(16, 256, 0, 1e-10, MU, eta, psi)
        dt = time.time() - t0
        extra["sap_gcr_32x64"] = {"s_per_rhs": dt, "status": st, "ifail": ifail,
                                  "rel_residual": rho / np.sqrt(eta.norm2()), "nkv": 16, "isolv": 1, "nmr": 4,
                                  "ncy": 5, "bs": list(BS), "res": 1e-10,
                                  "solver": "plain GPU sap_gcr: FP64 outer residual, FP32 SAP and Krylov space"}
        eta.free(); psi.free()
    s.free(); r.free()
    qb.release_workspace()

    if not args.no_solver and d.world == 1:
        # each workload reports its own failure instead of ending the run
        for key, fn in (("solver", solver_c3), ("batched", batched_c4), ("learned", learned_c5)):
            try:
                extra[key] = fn(qb)
            except Exception as e:
                extra[key] = {"error": repr(e)[:300]}
                try:
                    qb.release_workspace()
                except Exception:
                    pass
    cpu = None
    if not args.no_cpu_baseline and d.rank == 0 and d.world == 1 and L == LATTICE:
        try:
            cpu = cpu_reference_timing(check=(ipt, r_host, r32_host))
        except Exception as e:  # the baseline is reported, not required
            cpu = {"unavailable": str(e)[:200]}

    traffic = None
    pf = os.path.join(ROOT, "profiles", "dw_dble_traffic.json")
    if os.path.exists(pf):
        try:
            traffic = json.load(open(pf)).get("bytes_per_launch_full_lattice")
        except Exception:
            traffic = None

    if d.rank == 0:
        out = {
            "metric": "Dw_dble GB/s", "value": value, "unit": "GB/s", "n_gpus": d.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA if L == LATTICE else "synthetic (device-generated links exp(0.3 X), Gaussian source)",
            "config": bench_config(d.world) if L == LATTICE else {"workload": "Dw_dble profiling case",
                                                                  "lattice": list(L)},
            "roofline": {"bound": "hbm", "kernel": "dirac_staged_kernel<OP_SW|OP_HOP, all sites> (Dw_dble, SW staged)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_launch": bytes_step},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": args.steps,
        }
        out.update(extra)
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
