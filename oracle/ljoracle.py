"""ctypes bindings for the CPU oracle (libljoracle.so) and the reference harness
(_ref/libljref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker.  The product path never imports
this module.

The oracle restates the reference's cell-grid path (OptixLJ
Cuda-version/cudaLJ.cu) in C; see ljoracle.c for the line-by-line citations.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "libljoracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libljref.so")


class Grid(C.Structure):
    """Cell grid: origin, cell width and dims (x fastest), as ljo_grid."""

    _fields_ = [("origin", C.c_float * 3), ("width", C.c_float), ("dim", C.c_int * 3)]

    @property
    def ncells(self) -> int:
        return int(self.dim[0]) * int(self.dim[1]) * int(self.dim[2])

    def as_tuple(self):
        return (tuple(float(v) for v in self.origin), float(self.width), tuple(int(v) for v in self.dim))


_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _load():
    if not os.path.exists(_ORACLE_SO):
        raise RuntimeError(f"oracle library missing: {_ORACLE_SO} (run `make -C oracle`)")
    lib = C.CDLL(_ORACLE_SO)
    lib.ljo_srand48_state.restype = C.c_uint64
    lib.ljo_srand48_state.argtypes = [C.c_uint64]
    lib.ljo_drand48_fill.argtypes = [C.c_uint64, C.c_int64, _f64p]
    lib.ljo_generate_uniform.argtypes = [C.c_uint64, C.c_int64, _f32p, _f32p, _f32p, _f32p, _f32p]
    lib.ljo_generate_sphere.argtypes = [C.c_uint64, C.c_int64, _f32p, C.c_float, _f32p, _f32p, _f32p]
    lib.ljo_grid_from_box.restype = C.c_int
    lib.ljo_grid_from_box.argtypes = [_f32p, _f32p, C.c_float, C.POINTER(Grid)]
    lib.ljo_cells_of.argtypes = [C.POINTER(Grid), C.c_int64, _f32p, _f32p, _f32p, _i32p]
    lib.ljo_bin.restype = C.c_int
    lib.ljo_bin.argtypes = [C.POINTER(Grid), C.c_int64, _f32p, _f32p, _f32p, C.c_int, _i32p, _i32p, _i32p, _i32p]
    lib.ljo_count_candidates.restype = C.c_uint64
    lib.ljo_count_candidates.argtypes = [C.POINTER(Grid), _i32p]
    lib.ljo_lj_compat.restype = C.c_float
    lib.ljo_lj_compat.argtypes = [C.c_float] * 8
    lib.ljo_compat_energy.argtypes = [C.POINTER(Grid), C.c_int64, _f32p, _f32p, _f32p, _i32p, _i32p, _f32p]
    lib.ljo_config_forces.argtypes = [
        C.POINTER(Grid), C.c_int64, _f32p, _f32p, _f32p, _i32p, _i32p, C.c_float, C.c_float, C.c_float,
        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double),
        C.POINTER(C.c_double), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ljo_config_forces_f32_range.restype = C.c_uint64
    lib.ljo_config_forces_f32_range.argtypes = [
        C.POINTER(Grid), C.c_int64, C.c_int64, _f32p, _f32p, _f32p, _i32p, _i32p, C.c_float, C.c_float,
        C.c_float, _f32p, _f32p, C.c_int]
    lib.ljo_max_threads.restype = C.c_int
    lib.ljo_lj_compat_many.argtypes = [C.c_int64, _f32p, _f32p, _f32p]
    lib.ljo_brute_force.restype = C.c_uint64
    lib.ljo_brute_force.argtypes = [C.c_int64, _f32p, _f32p, _f32p, C.c_float, C.c_float, C.c_float, _f64p, _f64p]
    lib.ljo_pack_mixed.argtypes = [C.POINTER(Grid), C.c_int64, _f32p, _f32p, _i32p, _f32p, _f32p]
    lib.ljo_mixed_forces.argtypes = [
        C.POINTER(Grid), C.c_int64, C.c_int64, _f32p, _f32p, _f32p, _i32p, _i32p, C.c_float, C.c_float, C.c_float,
        C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p,
        C.c_void_p, C.c_void_p]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# --------------------------------------------------------------------- generation
def drand48_sequence(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, np.float64)
    lib().ljo_drand48_fill(seed, count, out)
    return out


def generate_uniform(seed: int, n: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    x, y, z = (np.empty(n, np.float32) for _ in range(3))
    lib().ljo_generate_uniform(seed, n, np.asarray(lo, np.float32), np.asarray(hi, np.float32), x, y, z)
    return x, y, z


def generate_sphere(seed: int, n: int, centre=(0.5, 0.5, 0.5), radius=1.0):
    x, y, z = (np.empty(n, np.float32) for _ in range(3))
    lib().ljo_generate_sphere(seed, n, np.asarray(centre, np.float32), radius, x, y, z)
    return x, y, z


# --------------------------------------------------------------------- grid / binning
def grid_from_box(lo, hi, cutoff) -> Grid:
    g = Grid()
    rc = lib().ljo_grid_from_box(np.asarray(lo, np.float32), np.asarray(hi, np.float32), cutoff, C.byref(g))
    if rc != 0:
        raise ValueError("invalid box or cutoff")
    return g


def cells_of(g: Grid, x, y, z) -> np.ndarray:
    out = np.empty(len(x), np.int32)
    lib().ljo_cells_of(C.byref(g), len(x), x, y, z, out)
    return out


@dataclass
class Binned:
    counts: np.ndarray
    offsets: np.ndarray
    perm: np.ndarray          # sorted slot -> original index
    cell_sorted: np.ndarray   # sorted slot -> cell id
    sx: np.ndarray
    sy: np.ndarray
    sz: np.ndarray


ORDER_INDEX = 0
ORDER_X = 1


def bin_particles(g: Grid, x, y, z, order: int = ORDER_X) -> Binned:
    n = len(x)
    counts = np.empty(g.ncells, np.int32)
    offsets = np.empty(g.ncells + 1, np.int32)
    perm = np.empty(n, np.int32)
    cs = np.empty(n, np.int32)
    if lib().ljo_bin(C.byref(g), n, x, y, z, order, counts, offsets, perm, cs) != 0:
        raise MemoryError("oracle binning failed")
    return Binned(counts, offsets, perm, cs, np.ascontiguousarray(x[perm]), np.ascontiguousarray(y[perm]),
                  np.ascontiguousarray(z[perm]))


def count_candidates(g: Grid, offsets) -> int:
    return int(lib().ljo_count_candidates(C.byref(g), offsets))


# --------------------------------------------------------------------- pair laws
def lj_compat(p1, p2, eps=1.0, sigma=1.0) -> float:
    return float(lib().ljo_lj_compat(*map(float, p1), *map(float, p2), eps, sigma))


def lj_compat_many(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Compat law for n pairs; a, b are (n, 3) float32 (self, other)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.empty(len(a), np.float32)
    lib().ljo_lj_compat_many(len(a), a.reshape(-1), b.reshape(-1), out)
    return out


def brute_force(x, y, z, rc: float, eps: float = 1.0, sigma: float | None = None):
    """All-pairs FP64 evaluation (input order): (pairs, e64[n], f64[n, 3])."""
    n = len(x)
    if sigma is None:
        sigma = float(np.float32(rc) / np.float32(2.5))
    e = np.empty(n, np.float64)
    f = np.empty((n, 3), np.float64)
    pairs = lib().ljo_brute_force(n, x, y, z, rc, eps, sigma, e, f)
    return int(pairs), e, f


def compat_energy(g: Grid, b: Binned) -> np.ndarray:
    v = np.empty(len(b.sx), np.float32)
    lib().ljo_compat_energy(C.byref(g), len(b.sx), b.sx, b.sy, b.sz, b.cell_sorted, b.offsets, v)
    return v


@dataclass
class ConfigResult:
    e32: np.ndarray | None
    f32: np.ndarray | None
    e64: np.ndarray | None
    f64: np.ndarray | None
    pairs: int
    etot: float
    virial: float
    escale: np.ndarray | None = None   # 4 eps sum_j (s^12 + s^6)        (FP64)
    fscale: np.ndarray | None = None   # 24 eps sum_j (2 s^12 + s^6) / r (FP64)
    nnb: np.ndarray | None = None      # interacting neighbours per particle

    def representable(self):
        """Particles whose FP64 energy, force and conditioning scales fit in float32 (FLT_MAX 3.4e38)."""
        lim = 1e38
        ok = np.abs(self.e64) < lim
        ok &= np.all(np.abs(self.f64) < lim, axis=1)
        if self.fscale is not None:
            ok &= (self.fscale < lim) & (self.escale < lim)
        return ok

    def scaled_tolerance(self, base: float = 1e-5):
        """Per-particle tolerance for float sums of m_i terms: max(base, 16 u sqrt(m_i)), u = 2^-24."""
        m = self.nnb if self.nnb is not None else np.ones(len(self.e64))
        return np.maximum(base, 16.0 * 2.0 ** -24 * np.sqrt(np.maximum(m, 1)))

    def force_errors(self, f, tol_base: float = 1e-5) -> dict:
        """Errors of a float force array (sorted order) against the FP64 result,
        over the particles whose FP64 results are representable in float."""
        f = np.asarray(f, np.float64).reshape(-1, 3)
        ok = self.representable()
        d = np.linalg.norm(f - self.f64, axis=1)[ok]
        f64 = self.f64[ok]
        fn = np.linalg.norm(f64, axis=1)
        nz = fn > 0
        rel = d[nz] / fn[nz]
        out = {"normwise": float(np.linalg.norm(f[ok] - f64) / max(np.linalg.norm(f64), 1e-300)),
               "max_rel": float(rel.max()) if rel.size else 0.0,
               "p99_rel": float(np.percentile(rel, 99)) if rel.size else 0.0,
               "excluded": int((~ok).sum())}
        if self.fscale is not None:
            sc = self.fscale[ok] > 0
            ratio = d[sc] / self.fscale[ok][sc]
            out["max_scaled"] = float(ratio.max()) if sc.any() else 0.0
            out["max_scaled_over_tol"] = float((ratio / self.scaled_tolerance(tol_base)[ok][sc]).max()) \
                if sc.any() else 0.0
        return out

    def energy_errors(self, e, tol_base: float = 1e-5) -> dict:
        e = np.asarray(e, np.float64)
        ok = self.representable()
        d = np.abs(e - self.e64)[ok]
        out = {"total_rel": float(abs(0.5 * e.sum() - self.etot) / max(abs(self.etot), 1e-300)),
               "excluded": int((~ok).sum())}
        if self.escale is not None:
            sc = self.escale[ok] > 0
            ratio = d[sc] / self.escale[ok][sc]
            out["max_scaled"] = float(ratio.max()) if sc.any() else 0.0
            out["max_scaled_over_tol"] = float((ratio / self.scaled_tolerance(tol_base)[ok][sc]).max()) \
                if sc.any() else 0.0
        return out


def config_forces(g: Grid, b: Binned, rc: float, eps: float = 1.0, sigma: float | None = None,
                  want32: bool = True, want64: bool = True) -> ConfigResult:
    n = len(b.sx)
    if sigma is None:
        sigma = float(np.float32(rc) / np.float32(2.5))
    e32 = np.empty(n, np.float32) if want32 else None
    f32 = np.empty((n, 3), np.float32) if want32 else None
    e64 = np.empty(n, np.float64) if want64 else None
    f64 = np.empty((n, 3), np.float64) if want64 else None
    es = np.empty(n, np.float64) if want64 else None
    fs = np.empty(n, np.float64) if want64 else None
    nnb = np.empty(n, np.int32)
    pairs = C.c_uint64(0)
    etot = C.c_double(0)
    vir = C.c_double(0)
    lib().ljo_config_forces(C.byref(g), n, b.sx, b.sy, b.sz, b.cell_sorted, b.offsets, rc, eps, sigma,
                            _ptr(e32), _ptr(f32), _ptr(e64), _ptr(f64), C.byref(pairs), C.byref(etot),
                            C.byref(vir), _ptr(es), _ptr(fs), _ptr(nnb))
    return ConfigResult(e32, f32, e64, f64, int(pairs.value), float(etot.value), float(vir.value), es, fs, nnb)


def config_forces_f32_range(g: Grid, b: Binned, k0: int, k1: int, rc: float, eps: float, sigma: float,
                            e32: np.ndarray, f32: np.ndarray, nthreads: int = 0) -> int:
    return int(lib().ljo_config_forces_f32_range(C.byref(g), k0, k1, b.sx, b.sy, b.sz, b.cell_sorted,
                                                 b.offsets, rc, eps, sigma, e32, f32, nthreads))


def max_threads() -> int:
    return int(lib().ljo_max_threads())


# --------------------------------------------------------------------- reference harness
def ref_available() -> bool:
    return os.path.exists(_REF_SO)


_ref = None


def ref_lib():
    """The reference's own code (cudaLJ.cu) built from source into _ref/libljref.so."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF_SO):
            raise RuntimeError(f"reference harness missing: {_REF_SO} (run `make -C oracle ref`)")
        r = C.CDLL(_REF_SO)
        r.ljref_lj_potential_host.restype = C.c_float
        r.ljref_lj_potential_host.argtypes = [C.c_float] * 8
        r.ljref_lj_potential_host_many.argtypes = [C.c_int64, _f32p, _f32p, _f32p]
        r.ljref_grid_dim.restype = C.c_int
        r.ljref_grid_dim.argtypes = [C.c_float, C.c_float]
        r.ljref_last_error.restype = C.c_int
        r.ljref_last_error.argtypes = [C.POINTER(C.c_int)]
        r.ljref_run.restype = C.c_int
        r.ljref_run.argtypes = [C.c_int, _f32p, _f32p, _f32p, C.c_float, C.c_float, _i32p, _i32p, _i32p,
                                _f32p, _f32p, _f32p, _i32p, _f32p, C.POINTER(C.c_ulonglong), _f32p, C.c_int]
        _ref = r
    return _ref


@dataclass
class RefRun:
    counts: np.ndarray
    prefix: np.ndarray
    cells: np.ndarray        # (ncells, 2): nbParticleInCell, offsetInContainer
    sx: np.ndarray
    sy: np.ndarray
    sz: np.ndarray
    index: np.ndarray
    v: np.ndarray
    nbinter: int
    stage_ms: np.ndarray     # count, scan, descriptors, scatter, candidates, pairs, binning span


def ref_run(x, y, z, box_width: float, cutoff: float, reps: int = 1) -> RefRun:
    """Runs the reference kernels (GPU) on injected positions.  Refuses, without
    launching, any position the reference kernels could not index."""
    r = ref_lib()
    n = len(x)
    G = r.ljref_grid_dim(box_width, cutoff)
    nc = G * G * G
    out = RefRun(np.empty(nc, np.int32), np.empty(nc + 1, np.int32), np.empty((nc, 2), np.int32),
                 np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.float32),
                 np.empty(n, np.int32), np.empty(n, np.float32), 0, np.empty(7, np.float32))
    nb = C.c_ulonglong(0)
    rc = r.ljref_run(n, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(y, np.float32),
                     np.ascontiguousarray(z, np.float32), box_width, cutoff, out.counts, out.prefix,
                     out.cells.reshape(-1), out.sx, out.sy, out.sz, out.index, out.v, C.byref(nb), out.stage_ms,
                     reps)
    if rc != 0:
        line = C.c_int(0)
        err = r.ljref_last_error(C.byref(line))
        raise RuntimeError(f"reference harness failed rc={rc} cuda_error={err} line={line.value}")
    out.nbinter = int(nb.value)
    return out


# --------------------------------------------------------------------- mixed precision
def pack_mixed(g: Grid, b: Binned):
    """binary16 y, z offsets (as float) of the sorted particles, as the GPU record pack."""
    n = len(b.sx)
    uy = np.empty(n, np.float32)
    uz = np.empty(n, np.float32)
    lib().ljo_pack_mixed(C.byref(g), n, b.sy, b.sz, b.cell_sorted, uy, uz)
    return uy, uz


def mixed_forces(g: Grid, b: Binned, uy, uz, rc: float, eps: float = 1.0, sigma: float | None = None,
                 k0: int = 0, k1: int | None = None) -> ConfigResult:
    """FP64 law on the stored (mixed) positions, targets [k0, k1), pairs chosen by the mixed test.
    Arrays of the result cover [k0, k1)."""
    n = len(b.sx)
    k1 = n if k1 is None else k1
    if sigma is None:
        sigma = float(np.float32(rc) / np.float32(2.5))
    e64 = np.zeros(n, np.float64)
    f64 = np.zeros((n, 3), np.float64)
    es = np.zeros(n, np.float64)
    fs = np.zeros(n, np.float64)
    nnb = np.zeros(n, np.int32)
    pairs = C.c_uint64(0)
    etot = C.c_double(0)
    vir = C.c_double(0)
    lib().ljo_mixed_forces(C.byref(g), k0, k1, b.sx, uy, uz, b.cell_sorted, b.offsets, rc, eps, sigma, _ptr(e64),
                           _ptr(f64), C.byref(pairs), C.byref(etot), C.byref(vir), _ptr(es), _ptr(fs), _ptr(nnb))
    sl = slice(k0, k1)
    return ConfigResult(None, None, e64[sl], f64[sl], int(pairs.value), float(etot.value), float(vir.value), es[sl],
                        fs[sl], nnb[sl])


# --------------------------------------------------------------------- spatial sort
def reorder(points: np.ndarray, radius: float) -> np.ndarray:
    """Restatement of the reference's reorder(N, points, radius)
    (SDK/optixMultiSphereAABB/sort.cu:29-41) and its key kernel count_per_cell
    (sort.cu:7-18): width = int(1.0f / radius) (:30); per point
    cell = int(x / radius) per axis, truncated (:12-14); id = cell_x +
    cell_y * width + cell_z * width * width (:15); .w = float(id) (:16); sort
    by .w ascending (:20-25, :38).  The division here is IEEE float32; the
    reference's own build (--use_fast_math) divides with the fast approximate
    division, which puts a coordinate lying within a couple of ulps of a cell
    face into the neighbouring cell now and then, so comparisons with this
    restatement use points away from the faces, and the reference's sort.cu
    built from source (sortref_keys, sortref_reorder) is the checker for the
    rest.  The integer id rounded once to float equals the reference's float
    sum as its compiler contracts it (fused multiply-adds).  Points of equal
    .w keep their input order (a stable sort): the reference's thrust::sort
    leaves that order unspecified, so comparisons against the reference
    itself use per-key sets.  Returns a new (n, 4) float32 array."""
    p = np.ascontiguousarray(points, dtype=np.float32)
    r = np.float32(radius)
    width = int(np.float32(1.0) / r)
    q = p[:, :3] / r
    c = np.trunc(q).astype(np.int64)
    ident = c[:, 0] + c[:, 1] * width + c[:, 2] * width * width
    w = ident.astype(np.int32).astype(np.float32)
    order = np.argsort(w, kind="stable")
    out = p[order].copy()
    out[:, 3] = w[order]
    return out


# --------------------------------------------------------------------- time step
def verlet_drift(xyz: np.ndarray, vel: np.ndarray, force: np.ndarray, dt: float, mass: float):
    """Half kick and drift of lj_step_verlet in single precision, one IEEE
    multiply and one add per update (numpy float32 arithmetic does not fuse):
    h = 0.5 * dt / mass; v' = v + h F; x' = x + dt v'.  The reference has no
    time step (its ParticlesContainer swap and cuRAND state, cudaLJ.cu:69-76
    and :96-97, anticipate one); this is the restatement the GPU step is
    checked against.  Returns (x', v', h), arrays (n, 3) float32."""
    h = np.float32(np.float32(0.5) * np.float32(dt) / np.float32(mass))
    v2 = (vel.astype(np.float32) + h * force.astype(np.float32)).astype(np.float32)
    x2 = (xyz.astype(np.float32) + np.float32(dt) * v2).astype(np.float32)
    return x2, v2, h


# --------------------------------------------------------------------- reference spatial sort
_SORTREF_SO = os.path.join(_HERE, "_ref", "libljsortref.so")
_sortref = None


def sortref_available() -> bool:
    return os.path.exists(_SORTREF_SO)


def _sortref_lib():
    """The reference's sort.cu (reorder, count_per_cell) built from source with its own flags into
    _ref/libljsortref.so (GPU)."""
    global _sortref
    if _sortref is None:
        if not os.path.exists(_SORTREF_SO):
            raise RuntimeError(f"reference sort harness missing: {_SORTREF_SO} (run `make -C oracle sortref`)")
        r = C.CDLL(_SORTREF_SO)
        r.ljsr_keys.restype = C.c_int
        r.ljsr_keys.argtypes = [C.c_int, _f32p, C.c_float, _f32p]
        r.ljsr_reorder.restype = C.c_int
        r.ljsr_reorder.argtypes = [C.c_int, _f32p, C.c_float]
        _sortref = r
    return _sortref


def sortref_keys(points: np.ndarray, radius: float) -> np.ndarray:
    """The reference's key (.w after count_per_cell) of each (n, 4) float32 point, input order."""
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
    keys = np.empty(len(pts), np.float32)
    rc = _sortref_lib().ljsr_keys(len(pts), pts.reshape(-1), radius, keys)
    if rc != 0:
        raise RuntimeError(f"reference count_per_cell failed: {rc}")
    return keys


def sortref_reorder(points: np.ndarray, radius: float) -> np.ndarray:
    """The reference's reorder(N, points, radius) on a copy of the (n, 4) float32 points."""
    pts = np.array(points, np.float32).reshape(-1, 4)
    rc = _sortref_lib().ljsr_reorder(len(pts), pts.reshape(-1), radius)
    if rc != 0:
        raise RuntimeError(f"reference reorder failed: {rc}")
    return pts
