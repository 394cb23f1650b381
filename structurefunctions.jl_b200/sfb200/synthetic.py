"""Seeded synthetic workloads with the shapes and value distributions of the benchmark configs.

No public dataset is involved: every input is generated here from a fixed seed (NumPy PCG64).

  c0  2D planar, N=4096, Float64, 32 Fourier modes (|k| in [1,64], amplitude |k|^-5/6) + N(0, 0.01^2)
      noise; L2SF; 32 log distance bins 1e-3..sqrt(2).
  c1  3D unit cube, N=65536, Float64, 64 solenoidal modes (|k| in [1,128], amplitude |k|^-11/6);
      L2SF, T2SF, L3SF, T3SF fused; 64 log bins 1e-4..sqrt(3).
  c2  sphere, N=200000 (lon, lat) degrees, Float32, radius 6371 km; 48 zonal/meridional modes
      (degree l in [1,200], amplitude l^-5/6, each component scaled to unit variance); L2SF along
      the arc; 48 log bins 1..20000 km.
  c3  2D planar, N=131072, Float32, field as c0; joint du_L histogram, 64 log distance bins
      1e-3..sqrt(2) x 256 linear value bins over [-5 sigma, 5 sigma], sigma = sqrt(2) std(u).
Log edges are materialized once as e_k = exp(ln(lo) + k (ln(hi) - ln(lo)) / nb) with the end points
set exactly.
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import operators as OP
from .bins import BinEdges, LinearBinEdges
from .metrics import Euclidean, Haversine


def log_edges(lo, hi, nb):
    k = np.arange(nb + 1, dtype=np.float64)
    e = np.exp(math.log(lo) + k * (math.log(hi) - math.log(lo)) / nb)
    e[0] = lo
    e[-1] = hi
    return e


def planar_field(x, n_modes, kmax, rng, noise_std):
    """Sum of random Fourier modes on [0,1)^2 (amplitude |k|^-5/6) plus Gaussian noise; x is (2, N)."""
    N = x.shape[1]
    kmag = rng.uniform(1.0, kmax, n_modes)
    th_k = rng.uniform(0.0, 2 * np.pi, n_modes)
    th_e = rng.uniform(0.0, 2 * np.pi, n_modes)
    phi = rng.uniform(0.0, 2 * np.pi, n_modes)
    amp = kmag ** (-5.0 / 6.0)
    kvec = np.stack([kmag * np.cos(th_k), kmag * np.sin(th_k)])  # (2, M)
    evec = np.stack([np.cos(th_e), np.sin(th_e)])                # (2, M)
    phase = 2 * np.pi * (kvec.T @ x) + phi[:, None]              # (M, N)
    u = evec @ (amp[:, None] * np.cos(phase))                    # (2, N)
    u += rng.normal(0.0, noise_std, size=(2, N))
    return u


def solenoidal_field(x, n_modes, kmax, rng):
    """64 random divergence-free modes in 3D (a_m perpendicular to k_m, |a_m| = |k|^-11/6)."""
    kmag = rng.uniform(1.0, kmax, n_modes)
    khat = rng.normal(size=(3, n_modes))
    khat /= np.linalg.norm(khat, axis=0)
    # an orthonormal pair perpendicular to k-hat, then a random angle in that plane
    ref = np.where(np.abs(khat[2]) < 0.9, np.array([[0.0], [0.0], [1.0]]), np.array([[1.0], [0.0], [0.0]]))
    e1 = np.cross(khat.T, ref.T).T
    e1 /= np.linalg.norm(e1, axis=0)
    e2 = np.cross(khat.T, e1.T).T
    ang = rng.uniform(0.0, 2 * np.pi, n_modes)
    avec = (np.cos(ang) * e1 + np.sin(ang) * e2) * kmag ** (-11.0 / 6.0)
    phi = rng.uniform(0.0, 2 * np.pi, n_modes)
    phase = 2 * np.pi * ((kmag * khat).T @ x) + phi[:, None]  # (M, N)
    return avec @ np.cos(phase)                                # (3, N)


def sphere_points(N, rng):
    lon = rng.uniform(-180.0, 180.0, N)
    lat = np.degrees(np.arcsin(rng.uniform(-1.0, 1.0, N)))
    return np.stack([lon, lat])


def sphere_field(x, n_modes, lmax, rng):
    """Zonal (u_east ~ cos(l lat)) and meridional (u_north ~ cos(l lon)) modes, unit variance."""
    lon = np.radians(x[0])
    lat = np.radians(x[1])
    N = x.shape[1]
    u = np.zeros((2, N))
    ls = rng.integers(1, lmax + 1, n_modes)
    phi = rng.uniform(0.0, 2 * np.pi, n_modes)
    for m in range(n_modes):
        a = float(ls[m]) ** (-5.0 / 6.0)
        if m % 2 == 0:
            u[0] += a * np.cos(ls[m] * lat + phi[m])
        else:
            u[1] += a * np.cos(ls[m] * lon + phi[m])
    u[0] /= u[0].std()
    u[1] /= u[1].std()
    return u


@dataclass
class Workload:
    name: str
    x: np.ndarray
    u: np.ndarray
    ops: tuple
    distance_bins: object
    metric: object = field(default_factory=Euclidean)
    value_bins: object = None
    flops_per_pair: int = 0
    sigma: float = float("nan")

    @property
    def n(self):
        return self.x.shape[1]

    @property
    def pairs(self):
        return self.n * (self.n - 1) // 2


def config(name, n=None):
    """Workload `name` in {"c0", "c1", "c2", "c3"} or one of the reference's own published GPU shapes
    {"r1d", "rjoint", "rsp1d", "rsp2d"}; `n` truncates to the first n points (same seed).

    r1d: 2D, N = 20000, Float32, L2SF, 32 linear bins LinearBinEdges(range(0, 0.3; length = 33)) -- the
    shape of the reference's A100 figures in gpu/SPEED_OF_LIGHT.md:37-45 and :680-686 (106.8 / 99.2
    bapps Float32, 60.2 bapps Float64); velocity field as c0.
    rjoint: the joint histogram at N = 20000, Float32, du_L on 64 linear value bins over +-5 sigma against
    the same 32 distance bins -- the size of gpu/SPEED_OF_LIGHT.md:291-298 (2.95 ms Float32, 4.51 ms
    Float64 on the A100); that document does not state the value axis, so this one is chosen.
    rsp1d: the one-dimensional single pass (the fused S2/L2/S3/L3 accumulation behind
    calculate_structure_functions_single_pass) on r1d's points and bins -- the shape of the "SP1D" rate
    of gpu/OPTIMAL_KERNEL_DESIGN.md:210-216 (43 G pairs/s on the A100, slices of 20000 points).
    rsp2d: the two-dimensional single pass at N = 20000, Float32, 50 linear distance bins over (0, 0.3]
    and one 50-bin value axis of +-5 sigma^2 shared by the six rows -- the shape of the "SP2D 50x50" rate
    of gpu/OPTIMAL_KERNEL_DESIGN.md:186,210-216 (28 G pairs/s on the A100, 64 slices of 20000 points),
    whose axes that document does not state either."""
    if name == "c0":
        N = 4096 if n is None else n
        rng = np.random.default_rng(0)
        x = rng.random((2, max(N, 4096)))
        u = planar_field(x, 32, 64.0, rng, 0.01)
        return Workload("c0 2D N=%d L2SF 32 log bins F64" % N, x[:, :N].copy(), u[:, :N].copy(), (OP.L2SF,),
                        BinEdges(log_edges(1e-3, math.sqrt(2.0), 32)), flops_per_pair=FLOPS["c0"])
    if name == "c1":
        N = 65536 if n is None else n
        rng = np.random.default_rng(1)
        x = rng.random((3, 65536))
        u = solenoidal_field(x, 64, 128.0, rng)
        return Workload("c1 3D N=%d L2/T2/L3/T3 64 log bins F64" % N, x[:, :N].copy(), u[:, :N].copy(),
                        (OP.L2SF, OP.T2SF, OP.L3SF, OP.T3SF), BinEdges(log_edges(1e-4, math.sqrt(3.0), 64)),
                        flops_per_pair=FLOPS["c1"])
    if name == "c2":
        N = 200000 if n is None else n
        rng = np.random.default_rng(2)
        x = sphere_points(200000, rng)
        u = sphere_field(x, 48, 200, rng)
        return Workload("c2 sphere N=%d L2SF 48 log bins 1..20000 km F32" % N,
                        x[:, :N].astype(np.float32), u[:, :N].astype(np.float32), (OP.L2SF,),
                        BinEdges(log_edges(1.0, 20000.0, 48)), metric=Haversine(6371.0),
                        flops_per_pair=FLOPS["c2"])
    if name == "c3":
        N = 131072 if n is None else n
        rng = np.random.default_rng(3)
        x = rng.random((2, 131072))
        u = planar_field(x, 32, 64.0, rng, 0.01)
        sigma = math.sqrt(2.0) * float(np.std(u.astype(np.float32).astype(np.float64).ravel()))
        vb = LinearBinEdges(-5.0 * sigma, 5.0 * sigma, 257)
        return Workload("c3 2D N=%d joint du_L 64x256 F32" % N, x[:, :N].astype(np.float32),
                        u[:, :N].astype(np.float32), (OP.ProjectedStructureFunctionType(1, 0),),
                        BinEdges(log_edges(1e-3, math.sqrt(2.0), 64)), value_bins=vb,
                        flops_per_pair=FLOPS["c3"], sigma=sigma)
    if name in ("r1d", "rjoint", "rsp1d"):
        N = 20000 if n is None else n
        rng = np.random.default_rng(5)
        x = rng.random((2, 20000))
        u = planar_field(x, 32, 64.0, rng, 0.01)
        dist = LinearBinEdges(0.0, 0.3, 33)
        if name == "r1d":
            return Workload("r1d 2D N=%d L2SF 32 linear bins (0, 0.3] F32" % N, x[:, :N].astype(np.float32),
                            u[:, :N].astype(np.float32), (OP.L2SF,), dist, flops_per_pair=FLOPS["r1d"])
        if name == "rsp1d":
            return Workload("rsp1d 2D N=%d single pass S2/L2/S3/L3 32 linear bins (0, 0.3] F32" % N,
                            x[:, :N].astype(np.float32), u[:, :N].astype(np.float32),
                            (OP.S2SF, OP.L2SF, OP.S3SF, OP.L3SF), dist, flops_per_pair=FLOPS["rsp1d"])
        sigma = math.sqrt(2.0) * float(np.std(u.astype(np.float32).astype(np.float64).ravel()))
        return Workload("rjoint 2D N=%d joint du_L 32x64 F32" % N, x[:, :N].astype(np.float32),
                        u[:, :N].astype(np.float32), (OP.ProjectedStructureFunctionType(1, 0),), dist,
                        value_bins=LinearBinEdges(-5.0 * sigma, 5.0 * sigma, 65), flops_per_pair=FLOPS["rjoint"],
                        sigma=sigma)
    if name == "rsp2d":
        from .single_pass import SINGLE_PASS_N, SinglePass2DRow  # (imports the API; kept out of module scope)

        N = 20000 if n is None else n
        rng = np.random.default_rng(6)
        x = rng.random((2, 20000))
        u = planar_field(x, 32, 64.0, rng, 0.01)
        sigma = math.sqrt(2.0) * float(np.std(u.astype(np.float32).astype(np.float64).ravel()))
        s2 = sigma * sigma
        return Workload("rsp2d 2D N=%d single pass 2D, six rows 50x50 F32" % N, x[:, :N].astype(np.float32),
                        u[:, :N].astype(np.float32), tuple(SinglePass2DRow(t) for t in range(SINGLE_PASS_N)),
                        LinearBinEdges(0.0, 0.3, 51), value_bins=LinearBinEdges(-5.0 * s2, 5.0 * s2, 51),
                        flops_per_pair=FLOPS["rsp2d"], sigma=sigma)
    raise KeyError(name)


def _serving_request(seed, k, n_min, n_max):
    """Request k of the serving workload (its own generator, seeded by (seed, k))."""
    rng = np.random.default_rng([seed, k])
    n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
    kind = int(rng.integers(0, 3))
    nb = int(rng.integers(32, 65))
    ops = (OP.L2SF,) if rng.random() < 0.5 else (OP.L3SF,)
    joint = rng.random() < 0.5
    if kind == 0:
        x = rng.random((2, n))
        u = planar_field(x, 32, 64.0, rng, 0.01)
        edges, metric = log_edges(1e-3, math.sqrt(2.0), nb), Euclidean()
    elif kind == 1:
        x = rng.random((3, n))
        u = solenoidal_field(x, 64, 128.0, rng)
        edges, metric = log_edges(1e-4, math.sqrt(3.0), nb), Euclidean()
    else:
        x = sphere_points(n, rng)
        u = sphere_field(x, 48, 200, rng).astype(np.float32)
        x = x.astype(np.float32)
        edges, metric = log_edges(1.0, 20000.0, nb), Haversine(6371.0)
    vb = None
    if joint:
        sigma = math.sqrt(2.0) * float(np.std(u.astype(np.float64)))
        vb = LinearBinEdges(-5.0 * sigma, 5.0 * sigma, 257)
    return {"x": x, "u": u, "ops": ops, "edges": edges, "metric": metric, "value_bins": vb,
            "kind": ("flat2", "flat3", "sphere")[kind], "n": n}


def _serving_chunk(args):
    seed, ks, n_min, n_max = args
    return [_serving_request(seed, k, n_min, n_max) for k in ks]


def serving_requests(count=2000, rate=200.0, seed=4, n_min=1000, n_max=100000, workers=0):
    """The batched-serving workload: `count` requests with Poisson arrivals (`rate` per second).

    Each request: N log-uniform in [n_min, n_max]; geometry uniformly 2D planar (c0's field), 3D
    planar (c1's field) or spherical (c2's field, Float32); 32-64 log distance bins over the geometry's
    range; order 2 or 3 (L2SF or L3SF); half of them also ask for the joint du_L histogram with 256
    linear value bins over [-5 sigma, 5 sigma]. Request k draws from its own generator (seed, k), so
    the set does not depend on `workers` (processes generating in parallel; 0 = in this process).
    Returns a list of dicts with keys `t` (arrival, seconds), `x`, `u`, `ops`, `edges`, `metric`,
    `value_bins` (None or LinearBinEdges), `kind`, `n`.
    """
    arrivals = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, count))
    if workers and workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp

        chunks = [list(range(a, min(a + 25, count))) for a in range(0, count, 25)]
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
            reqs = [r for part in pool.map(_serving_chunk, [(seed, c, n_min, n_max) for c in chunks]) for r in part]
    else:
        reqs = [_serving_request(seed, k, n_min, n_max) for k in range(count)]
    for r, t in zip(reqs, arrivals):
        r["t"] = float(t)
    return reqs


# Algorithmic flops per pair: the reference's FP64 formula as restated by the oracle, counting +, -,
# x, / and sqrt as 1, FMA as 2, one add per accumulated sum; binning compares and recheck work are
# not counted. These are the roofline numerators.
#   c0 (2D L2):  dx 2, r^2 3, du 2, p 3, p^2/r^2 2, acc 1                                   = 13
#   c1 (3D L2,T2,L3,T3): dx 3, r^2 5, du 3, p 5, |du|^2 5, L2 2, T2 1, sqrt 1, r_hat 3,
#        du.r_hat 5, L3 2, n_hat 6, du.n_hat 5, T3 2, acc 4                                 = 52
#   c2 (sphere L2, per-point basis precomputed): geodesic frame, tangents and increments 107,
#        plus 1 atan2 and 2 square roots counted as 1 each                                  = 110
#   c3 (2D joint du_L): dx 2, r^2 3, sqrt 1, r_hat 2, du 2, dot 3, L 1, acc 1                = 15
#   r1d, rjoint: as c0 and c3 (sqrt 1 added to r1d for the linear bins' key)             = 14, 15
#   rsp1d (S2, L2, S3, L3 of one pair, serial_single_pass.jl:151-400): dx 2, r^2 3, du 2,
#         inv(sqrt) 2, du_L 4, |du|^2 3, L2 / S3 / L3 3, acc 4                              = 23
#   rsp2d (six rows of one pair, serial_single_pass.jl:886-905): dx 2, r^2 3, du 2, inv(sqrt) 2,
#         du_L 4, |du|^2 3, L2 / T2 / S3 / L3 / L1T2 5, acc 6                               = 27
FLOPS = {"c0": 13, "c1": 52, "c2": 110, "c3": 15, "r1d": 14, "rjoint": 15, "rsp1d": 23, "rsp2d": 27}

# Operations per pair of the mixed kernel's own formulation (FP64 + FP32, same counting), for
# reference next to FLOPS:
#   c0: dx 2, r^2 3, du 2, p 3, rsqrt 1, L 1, L^2 1, acc 1                                  = 14
#   c1: dx 3, r^2 5, du 3, p 5, cz 3, |du|^2 5, c2 3, rsqrt 2, L 1, T 1, T2 2, L2 1, L3 1,
#       T3 2, acc 4                                                                        = 41
#   c2: d 3, s 3, |d|^2 5, |s|^2 5, dU 3, d.dU 5, scale 3, rsqrt 1, L 1, L^2 1, acc 1        = 31
#   c3: dx 2, r^2 3, du 2, p 3, rsqrt 1, L 1, t 2, centre 1, acc 1                           = 16
#   rsp1d: dx 2, r^2 3, du 2, p 3, |du|^2 3, rsqrt 1, L 1, L^2 1, S3 1, L3 1, acc 4        = 22
#          (S2 is |du|^2 itself)
KERNEL_FLOPS = {"c0": 14, "c1": 41, "c2": 31, "c3": 16, "r1d": 15, "rjoint": 16, "rsp1d": 22}
