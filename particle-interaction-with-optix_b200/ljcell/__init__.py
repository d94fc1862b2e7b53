"""ljcell -- Python host layer over the C ABI of the B200 cell-grid LJ path.

This mirrors the reference's step (OptixLJ Cuda-version/cudaLJ.cu,
executeSimulation at cudaLJ.cu:515-677): generation, the cell-grid build
(count, scan, descriptors, scatter), the candidate count and the pair
kernel, each a call into libljcell.so (include/ljcell.h).  PyTorch provides
device memory and streams only; every computation runs in the library's own
sm_100a kernels.  There is no CPU fallback: importing this package on a
machine where libljcell.so cannot be loaded raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# LJCELL_CHECKS=1 loads the bounds-checked debug build (compiled with -DLJ_CHECKS) instead
LIB_PATH = os.path.join(_HERE, "libljcell_checks.so" if os.environ.get("LJCELL_CHECKS") == "1" else "libljcell.so")

LJ_OK, LJ_EINVAL, LJ_ENOMEM, LJ_ECUDA, LJ_ETIMEOUT, LJ_ERANGE, LJ_EUNSUPPORTED, LJ_ECHECK = range(8)
ORDER_INDEX = 0
ORDER_X = 1


class Grid(C.Structure):
    """lj_grid: origin, cell width, dims (x fastest)."""

    _fields_ = [("origin", C.c_float * 3), ("width", C.c_float), ("dim", C.c_int * 3)]

    @property
    def ncells(self) -> int:
        return int(self.dim[0]) * int(self.dim[1]) * int(self.dim[2])

    def __repr__(self):
        return (f"Grid(origin={tuple(self.origin)}, width={self.width}, dim={tuple(self.dim)})")


class Params(C.Structure):
    """lj_params: truncated LJ cutoff, epsilon, sigma."""

    _fields_ = [("cutoff", C.c_float), ("epsilon", C.c_float), ("sigma", C.c_float)]


class Totals(C.Structure):
    """lj_totals: E = 1/2 sum e_i, virial, interacting ordered pairs."""

    _fields_ = [("energy", C.c_double), ("virial", C.c_double), ("pairs", C.c_ulonglong), ("pad", C.c_ulonglong)]


class Particles(C.Structure):
    """lj_particles == ParticlesContainer<float> (cudaLJ.cu:60-67)."""

    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("v", C.c_void_p),
                ("index", C.c_void_p), ("nbParticles", C.c_int)]


class Tuning(C.Structure):
    """lj_tuning: implementation choices (pair_kernel 0 default, 1 one target per thread with windows in
    shared memory, 6 row passes, 10 row passes with two targets per lane, 11 as 1 with whole rows, 12
    targets paired inside their cell over whole rows; the retired values 2-5 and 7-9 run the kernel of
    their family)."""

    _fields_ = [("pair_kernel", C.c_int), ("scatter_passes", C.c_int), ("reserved", C.c_int * 6)]


class System(C.Structure):
    """lj_system: box, truncated-law parameters and particle range of one system of a batch."""

    _fields_ = [("lo", C.c_float * 3), ("hi", C.c_float * 3), ("params", Params), ("first", C.c_int),
                ("n", C.c_int)]


class BatchConfig(C.Structure):
    """lj_batch_config: cell-width multiple, CTA size and targets per thread of the batched step."""

    _fields_ = [("cell_multiple", C.c_float), ("threads", C.c_int), ("per_thread", C.c_int),
                ("reserved", C.c_int * 5)]


class LJError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: {status_str(status)} (status {status})")
        self.status = status


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libljcell.so not built at {LIB_PATH}; run __graft_entry__.build() or "
                          f"`make -C particle-interaction-with-optix_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    vp, i32, i64, f32 = C.c_void_p, C.c_int, C.c_longlong, C.c_float
    f3 = C.POINTER(C.c_float)
    sig = {
        "lj_abi_version": (C.c_int, []),
        "lj_status_str": (C.c_char_p, [i32]),
        "lj_create": (i32, [C.POINTER(vp), i32, vp]),
        "lj_destroy": (i32, [vp]),
        "lj_set_stream": (i32, [vp, vp]),
        "lj_sync": (i32, [vp]),
        "lj_generate_uniform": (i32, [vp, C.c_uint64, i32, f3, f3, C.POINTER(Particles), vp]),
        "lj_generate_sphere": (i32, [vp, C.c_uint64, i32, f3, f32, C.POINTER(Particles), vp]),
        "lj_grid_from_box": (i32, [f3, f3, f32, C.POINTER(Grid)]),
        "lj_grid_compat": (i32, [f32, f32, C.POINTER(Grid)]),
        "lj_count_cells": (i32, [vp, C.POINTER(Grid), i32, vp, vp, vp, i32, vp]),
        "lj_exclusive_scan": (i32, [vp, vp, i64, vp]),
        "lj_exclusive_scan_noalloc": (i32, [vp, i64, vp, vp]),
        "lj_cell_descriptors": (i32, [vp, vp, i64, vp]),
        "lj_bin": (i32, [vp, C.POINTER(Grid), i32, vp, vp, vp, i32, i32, vp, vp, vp, C.POINTER(Particles), vp, vp]),
        "lj_count_candidates": (i32, [vp, C.POINTER(Grid), vp, vp]),
        "lj_compute_compat": (i32, [vp, C.POINTER(Grid), i32, vp, vp, vp, vp]),
        "lj_compute": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, i32, vp, vp, vp]),
        "lj_set_tuning": (i32, [vp, C.POINTER(Tuning)]),
        "lj_get_tuning": (i32, [vp, C.POINTER(Tuning)]),
        "lj_autotune_compute": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, C.POINTER(i32),
                                      C.POINTER(C.c_float)]),
        "lj_batch_create": (i32, [vp, i32, C.POINTER(System), C.POINTER(BatchConfig), C.POINTER(vp)]),
        "lj_batch_destroy": (i32, [vp]),
        "lj_batch_get_config": (i32, [vp, C.POINTER(BatchConfig)]),
        "lj_batch_grid": (i32, [vp, i32, C.POINTER(Grid)]),
        "lj_batch_run": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "lj_batch_run_graph": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "lj_batch_run_separate": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "lj_batch_autotune": (i32, [vp, vp, vp, vp, vp, C.POINTER(BatchConfig), C.POINTER(C.c_float)]),
        "lj_pack_mixed": (i32, [vp, C.POINTER(Grid), i32, vp, vp, vp]),
        "lj_compute_mixed": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, vp, vp, vp]),
        "lj_test_scan_withheld_tile": (i32, [vp, vp, i64, vp]),
        "lj_test_scan_noalloc_withheld_tile": (i32, [vp, i64, vp, vp]),
        "lj_compute_half": (i32, [vp, vp, vp, i32, vp, vp, vp, vp, vp]),
        "lj_compute_range": (i32, [vp, vp, vp, i32, vp, vp, vp, i32, i32, i32, vp, vp, vp]),
        "lj_reorder": (i32, [vp, i32, vp, C.c_float]),
        "lj_step_verlet": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, C.c_float, C.c_float, vp, vp, vp, vp,
                                 vp, vp, vp, vp]),
        "lj_simulate_host": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, vp, vp, vp,
                                   C.POINTER(Totals)]),
        "lj_simulate_host_async": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, vp, vp, vp,
                                   C.POINTER(Totals)]),
        "lj_simulate_host_wait": (i32, [vp]),
        "lj_select_layers": (i32, [vp, C.POINTER(Grid), i32, vp, i32, i32, vp, vp, vp]),
        "lj_test_fail_alloc": (i32, [i32]),
        "lj_simulate_host_inorder_async": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, vp, vp,
                                           C.POINTER(Totals)]),
        "lj_simulate_host_inorder": (i32, [vp, C.POINTER(Grid), C.POINTER(Params), i32, vp, vp, vp, vp, vp,
                                     C.POINTER(Totals)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = _load()
ABI_SYMBOLS = ("lj_abi_version", "lj_status_str", "lj_create", "lj_destroy", "lj_set_stream", "lj_sync",
               "lj_generate_uniform", "lj_generate_sphere", "lj_grid_from_box", "lj_grid_compat",
               "lj_count_cells", "lj_exclusive_scan", "lj_exclusive_scan_noalloc", "lj_cell_descriptors", "lj_bin", "lj_count_candidates",
               "lj_compute_compat", "lj_compute", "lj_set_tuning", "lj_get_tuning", "lj_autotune_compute", "lj_batch_create",
               "lj_batch_destroy", "lj_batch_get_config", "lj_batch_grid", "lj_batch_run", "lj_batch_run_graph",
               "lj_batch_run_separate", "lj_batch_autotune", "lj_pack_mixed", "lj_compute_mixed",
               "lj_test_scan_withheld_tile", "lj_test_scan_noalloc_withheld_tile", "lj_compute_half", "lj_compute_range", "lj_reorder", "lj_step_verlet", "lj_simulate_host",
               "lj_simulate_host_async", "lj_simulate_host_wait", "lj_simulate_host_inorder_async",
               "lj_simulate_host_inorder", "lj_select_layers", "lj_test_fail_alloc")


def lib() -> C.CDLL:
    return _lib


def status_str(s: int) -> str:
    return _lib.lj_status_str(s).decode()


def _check(s: int, where: str):
    if s != LJ_OK:
        raise LJError(s, where)


def _f3(v):
    return (C.c_float * 3)(*[float(a) for a in v])


def grid_from_box(lo, hi, cutoff: float) -> Grid:
    g = Grid()
    _check(_lib.lj_grid_from_box(_f3(lo), _f3(hi), cutoff, C.byref(g)), "lj_grid_from_box")
    return g


def grid_compat(box_width: float, cutoff: float) -> Grid:
    g = Grid()
    _check(_lib.lj_grid_compat(box_width, cutoff, C.byref(g)), "lj_grid_compat")
    return g


def default_sigma(cutoff: float) -> float:
    """sigma = r_c / 2.5 evaluated in float32."""
    return float(np.float32(cutoff) / np.float32(2.5))


def test_fail_alloc(k: int):
    """lj_test_fail_alloc: make the k-th next scratch growth fail with LJ_ENOMEM (0: off)."""
    _check(_lib.lj_test_fail_alloc(int(k)), "lj_test_fail_alloc")


def exclusive_scan_noalloc(counts, offsets, stream=None):
    """lj_exclusive_scan_noalloc: the scan without a context or any device
    allocation (scratch is a fixed array inside the library).  `counts` and
    `offsets` are int32 CUDA tensors (offsets has counts.numel() + 1 entries)."""
    s = None if stream is None else C.c_void_p(stream.cuda_stream)
    _check(_lib.lj_exclusive_scan_noalloc(_ptr(counts), int(counts.numel()), _ptr(offsets), s),
           "lj_exclusive_scan_noalloc")
    return offsets


def params(cutoff: float, epsilon: float = 1.0, sigma: float | None = None) -> Params:
    return Params(cutoff, epsilon, default_sigma(cutoff) if sigma is None else sigma)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


@dataclass
class Binned:
    """Device buffers of one binned system (torch tensors)."""
    n: int
    order: int
    counts: object
    offsets: object
    xyzi: object           # (n, 4) float32: x, y, z, original index bits
    cell: object           # (n,) int32
    sx: object | None = None
    sy: object | None = None
    sz: object | None = None
    index: object | None = None
    cells: object | None = None   # (ncells, 2) int32 CellDescriptor view


class Context:
    """An lj_ctx bound to one device and one stream."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        s = None if stream is None else C.c_void_p(stream.cuda_stream)
        _check(_lib.lj_create(C.byref(h), device, s), "lj_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.lj_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream):
        _check(_lib.lj_set_stream(self._h, None if stream is None else C.c_void_p(stream.cuda_stream)),
               "lj_set_stream")

    def sync(self):
        _check(_lib.lj_sync(self._h), "lj_sync")

    def set_tuning(self, pair_kernel: int = 0, scatter_passes: int = 0):
        t = Tuning()
        t.pair_kernel = pair_kernel
        t.scatter_passes = scatter_passes
        _check(_lib.lj_set_tuning(self._h, C.byref(t)), "lj_set_tuning")

    def autotune_compute(self, g: Grid, p: Params, b: Binned):
        """Times pair kernels 1, 6, 10, 11 and 12 on these binned particles and keeps the fastest."""
        k = C.c_int(0)
        ms = C.c_float(0)
        _check(_lib.lj_autotune_compute(self._h, C.byref(g), C.byref(p), b.n, _ptr(b.xyzi), _ptr(b.cell),
                                        _ptr(b.offsets), C.byref(k), C.byref(ms)), "lj_autotune_compute")
        return int(k.value), float(ms.value)

    def get_tuning(self) -> dict:
        t = Tuning()
        _check(_lib.lj_get_tuning(self._h, C.byref(t)), "lj_get_tuning")
        return {"pair_kernel": t.pair_kernel, "scatter_passes": t.scatter_passes}

    # ------------------------------------------------------------ generation
    def _gen_out(self, n, want_soa, want_aos):
        t = self.torch
        soa = None
        if want_soa:
            soa = {k: t.empty(n, dtype=t.float32, device=self.device) for k in ("x", "y", "z", "v")}
            soa["index"] = t.empty(n, dtype=t.int32, device=self.device)
        aos = t.empty((n, 3), dtype=t.float32, device=self.device) if want_aos else None
        p = Particles()
        if soa:
            p.x, p.y, p.z, p.v, p.index = (soa[k].data_ptr() for k in ("x", "y", "z", "v", "index"))
        p.nbParticles = n
        return soa, aos, p

    def generate_uniform(self, seed: int, n: int, lo=(0, 0, 0), hi=(1, 1, 1), soa=True, aos=False):
        s, a, p = self._gen_out(n, soa, aos)
        _check(_lib.lj_generate_uniform(self._h, seed, n, _f3(lo), _f3(hi), C.byref(p), _ptr(a)),
               "lj_generate_uniform")
        return s, a

    def generate_sphere(self, seed: int, n: int, centre=(0.5, 0.5, 0.5), radius=1.0, soa=True, aos=False):
        s, a, p = self._gen_out(n, soa, aos)
        _check(_lib.lj_generate_sphere(self._h, seed, n, _f3(centre), radius, C.byref(p), _ptr(a)),
               "lj_generate_sphere")
        return s, a

    # ------------------------------------------------------------ binning
    def alloc_binned(self, g: Grid, n: int, order: int = ORDER_X, soa: bool = False, cells: bool = False) -> Binned:
        t = self.torch
        dev = self.device
        b = Binned(n, order, t.empty(g.ncells, dtype=t.int32, device=dev),
                   t.empty(g.ncells + 1, dtype=t.int32, device=dev),
                   t.empty((max(n, 1), 4), dtype=t.float32, device=dev),
                   t.empty(max(n, 1), dtype=t.int32, device=dev))
        if soa:
            b.sx, b.sy, b.sz = (t.empty(max(n, 1), dtype=t.float32, device=dev) for _ in range(3))
            b.index = t.empty(max(n, 1), dtype=t.int32, device=dev)
        if cells:
            b.cells = t.empty((g.ncells, 2), dtype=t.int32, device=dev)
        return b

    def bin(self, g: Grid, x, y, z, stride: int = 1, order: int = ORDER_X, out: Binned | None = None,
            soa: bool = False, cells: bool = False) -> Binned:
        n = int(x.numel()) // stride if stride > 1 else int(x.numel())
        b = out if out is not None else self.alloc_binned(g, n, order, soa, cells)
        b.order = order
        sp = None
        if b.sx is not None or b.index is not None:
            sp = Particles(None if b.sx is None else b.sx.data_ptr(), None if b.sy is None else b.sy.data_ptr(),
                           None if b.sz is None else b.sz.data_ptr(), None,
                           None if b.index is None else b.index.data_ptr(), n)
        _check(_lib.lj_bin(self._h, C.byref(g), n, _ptr(x), _ptr(y), _ptr(z), stride, order, _ptr(b.counts),
                           _ptr(b.offsets), _ptr(b.cells), C.byref(sp) if sp is not None else None, _ptr(b.xyzi),
                           _ptr(b.cell)), "lj_bin")
        return b

    def count_cells(self, g: Grid, x, y, z, stride: int = 1, counts=None):
        t = self.torch
        n = int(x.numel()) // stride if stride > 1 else int(x.numel())
        counts = counts if counts is not None else t.empty(g.ncells, dtype=t.int32, device=self.device)
        _check(_lib.lj_count_cells(self._h, C.byref(g), n, _ptr(x), _ptr(y), _ptr(z), stride, _ptr(counts)),
               "lj_count_cells")
        return counts

    def exclusive_scan(self, counts, offsets=None):
        t = self.torch
        nc = int(counts.numel())
        offsets = offsets if offsets is not None else t.empty(nc + 1, dtype=t.int32, device=self.device)
        _check(_lib.lj_exclusive_scan(self._h, _ptr(counts), nc, _ptr(offsets)), "lj_exclusive_scan")
        return offsets

    def cell_descriptors(self, offsets, cells=None):
        t = self.torch
        nc = int(offsets.numel()) - 1
        cells = cells if cells is not None else t.empty((nc, 2), dtype=t.int32, device=self.device)
        _check(_lib.lj_cell_descriptors(self._h, _ptr(offsets), nc, _ptr(cells)), "lj_cell_descriptors")
        return cells

    # ------------------------------------------------------------ interactions
    def count_candidates(self, g: Grid, offsets, out=None):
        t = self.torch
        out = out if out is not None else t.empty(1, dtype=t.int64, device=self.device)
        _check(_lib.lj_count_candidates(self._h, C.byref(g), _ptr(offsets), _ptr(out)), "lj_count_candidates")
        return out

    def compute_compat(self, g: Grid, b: Binned, v=None):
        t = self.torch
        v = v if v is not None else t.empty(max(b.n, 1), dtype=t.float32, device=self.device)
        _check(_lib.lj_compute_compat(self._h, C.byref(g), b.n, _ptr(b.xyzi), _ptr(b.cell), _ptr(b.offsets),
                                      _ptr(v)), "lj_compute_compat")
        return v

    def alloc_outputs(self, n: int):
        t = self.torch
        e = t.empty(max(n, 1), dtype=t.float32, device=self.device)
        f = t.empty((max(n, 1), 3), dtype=t.float32, device=self.device)
        tot = t.zeros(4, dtype=t.float64, device=self.device)  # one lj_totals (32 bytes)
        return e, f, tot

    def compute(self, g: Grid, p: Params, b: Binned, energy=None, force=None, totals=None, want_energy=True,
                want_force=True):
        if energy is None and force is None and totals is None:
            energy, force, totals = self.alloc_outputs(b.n)
        _check(_lib.lj_compute(self._h, C.byref(g), C.byref(p), b.n, _ptr(b.xyzi), _ptr(b.cell), _ptr(b.offsets),
                               b.order, _ptr(energy) if want_energy else None,
                               _ptr(force) if want_force else None, _ptr(totals)), "lj_compute")
        return energy, force, totals

    def compute_range(self, g: Grid, p: Params, b: Binned, kb: int, ke: int, energy=None, force=None, totals=None):
        """lj_compute_range: the truncated law for the sorted targets [kb, ke) only."""
        if energy is None and force is None and totals is None:
            energy, force, totals = self.alloc_outputs(b.n)
        _check(_lib.lj_compute_range(self._h, C.byref(g), C.byref(p), b.n, _ptr(b.xyzi), _ptr(b.cell),
                                     _ptr(b.offsets), b.order, int(kb), int(ke), _ptr(energy), _ptr(force),
                                     _ptr(totals)), "lj_compute_range")
        return energy, force, totals

    def select_layers(self, g: Grid, xyz, layer_lo: int, layer_hi: int):
        """lj_select_layers: the rows of the (m, 3) float32 device tensor xyz whose z layer is layer_lo,
        and those whose z layer is layer_hi, in input order (a negative layer selects nothing).
        Synchronises to read the two counts."""
        t = self.torch
        m = int(xyz.shape[0])
        xyz = xyz.contiguous()
        out_lo = t.empty((max(m, 1), 3), dtype=t.float32, device=self.device)
        out_hi = t.empty((max(m, 1), 3), dtype=t.float32, device=self.device)
        counts = t.zeros(2, dtype=t.int32, device=self.device)
        _check(_lib.lj_select_layers(self._h, C.byref(g), m, _ptr(xyz), int(layer_lo), int(layer_hi), _ptr(out_lo),
                                     _ptr(out_hi), _ptr(counts)), "lj_select_layers")
        c_lo, c_hi = counts.tolist()
        return out_lo[:c_lo], out_hi[:c_hi]

    def compute_half(self, g: Grid, p: Params, b: Binned, energy=None, force=None, totals=None):
        """lj_compute_half: the truncated law with each unordered pair evaluated once (any order)."""
        if energy is None and force is None and totals is None:
            energy, force, totals = self.alloc_outputs(b.n)
        _check(_lib.lj_compute_half(self._h, C.byref(g), C.byref(p), b.n, _ptr(b.xyzi), _ptr(b.offsets),
                                    _ptr(energy), _ptr(force), _ptr(totals)), "lj_compute_half")
        return energy, force, totals

    def pack_mixed(self, g: Grid, b: Binned, rec=None):
        """Mixed-precision records (n, 2) float32: x and the binary16 pair (uy, uz) bit-packed."""
        t = self.torch
        rec = rec if rec is not None else t.empty((max(b.n, 1), 2), dtype=t.float32, device=self.device)
        _check(_lib.lj_pack_mixed(self._h, C.byref(g), b.n, _ptr(b.xyzi), _ptr(b.cell), _ptr(rec)), "lj_pack_mixed")
        return rec

    def compute_mixed(self, g: Grid, p: Params, b: Binned, rec, energy=None, force=None, totals=None):
        if energy is None and force is None and totals is None:
            energy, force, totals = self.alloc_outputs(b.n)
        _check(_lib.lj_compute_mixed(self._h, C.byref(g), C.byref(p), b.n, _ptr(rec), _ptr(b.cell), _ptr(b.offsets),
                                     _ptr(energy), _ptr(force), _ptr(totals)), "lj_compute_mixed")
        return energy, force, totals

    def reorder(self, points, radius: float):
        """lj_reorder: sorts the (n, 4) float32 device tensor `points` in place by cell key (stored in
        column 3), as the reference's reorder(N, points, radius)."""
        n = int(points.shape[0]) if points.numel() else 0
        _check(_lib.lj_reorder(self._h, n, _ptr(points), C.c_float(radius)), "lj_reorder")
        return points

    def step_verlet(self, g: Grid, p: Params, b: Binned, vel, force, dt: float, mass: float = 1.0, energy=None,
                    totals=None):
        """lj_step_verlet: one velocity-Verlet step of the binned system b (LJ_ORDER_X) in place: b.xyzi,
        b.cell, b.counts, b.offsets, vel (n, 3) and force (n, 3) hold the new sorted state afterwards."""
        _check(_lib.lj_step_verlet(self._h, C.byref(g), C.byref(p), b.n, C.c_float(dt), C.c_float(mass),
                                   _ptr(b.xyzi), _ptr(vel), _ptr(force), _ptr(b.cell), _ptr(b.counts),
                                   _ptr(b.offsets), _ptr(energy), _ptr(totals)), "lj_step_verlet")
        return b

    def simulate_host(self, g: Grid, p: Params, hx: np.ndarray, hy: np.ndarray, hz: np.ndarray,
                      energy: np.ndarray | None = None, force: np.ndarray | None = None,
                      index: np.ndarray | None = None):
        n = len(hx)
        tot = Totals()
        fp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        _check(_lib.lj_simulate_host(self._h, C.byref(g), C.byref(p), n, fp(hx), fp(hy), fp(hz), fp(energy),
                                     fp(force), fp(index), C.byref(tot)), "lj_simulate_host")
        return tot

    def simulate_host_async(self, g: Grid, p: Params, hx: np.ndarray, hy: np.ndarray, hz: np.ndarray,
                            energy: np.ndarray | None = None, force: np.ndarray | None = None,
                            index: np.ndarray | None = None, totals=None):
        """lj_simulate_host_async: queues one host-buffer step and returns; the arrays (pinned for the
        copies to overlap) and the returned Totals must stay alive and untouched until
        simulate_host_wait()."""
        n = len(hx)
        tot = totals if totals is not None else Totals()
        fp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        # the library writes into these at lj_simulate_host_wait: keep them alive until then
        if not hasattr(self, "_pending"):
            self._pending = []
        self._pending.append((tot, hx, hy, hz, energy, force, index))
        _check(_lib.lj_simulate_host_async(self._h, C.byref(g), C.byref(p), n, fp(hx), fp(hy), fp(hz), fp(energy),
                                           fp(force), fp(index), C.byref(tot)), "lj_simulate_host_async")
        return tot

    def simulate_host_inorder_async(self, g: Grid, p: Params, hx: np.ndarray, hy: np.ndarray, hz: np.ndarray,
                                    energy: np.ndarray | None = None, force: np.ndarray | None = None, totals=None):
        """lj_simulate_host_inorder_async: as simulate_host_async with energy and force in the input order
        (no index); completed by simulate_host_wait()."""
        n = len(hx)
        tot = totals if totals is not None else Totals()
        fp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        if not hasattr(self, "_pending"):
            self._pending = []
        self._pending.append((tot, hx, hy, hz, energy, force))
        _check(_lib.lj_simulate_host_inorder_async(self._h, C.byref(g), C.byref(p), n, fp(hx), fp(hy), fp(hz),
                                                   fp(energy), fp(force), C.byref(tot)),
               "lj_simulate_host_inorder_async")
        return tot

    def simulate_host_inorder(self, g: Grid, p: Params, hx: np.ndarray, hy: np.ndarray, hz: np.ndarray,
                              energy: np.ndarray | None = None, force: np.ndarray | None = None):
        """lj_simulate_host_inorder: one host-buffer step, energy and force in the input order."""
        tot = Totals()
        fp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        try:
            _check(_lib.lj_simulate_host_inorder(self._h, C.byref(g), C.byref(p), len(hx), fp(hx), fp(hy), fp(hz),
                                                 fp(energy), fp(force), C.byref(tot)), "lj_simulate_host_inorder")
        finally:
            self._pending = []
        return tot

    def simulate_host_wait(self):
        try:
            _check(_lib.lj_simulate_host_wait(self._h), "lj_simulate_host_wait")
        finally:
            self._pending = []


def totals_from_tensor(tot) -> dict:
    """Decodes one lj_totals held in a 4-element float64 tensor."""
    raw = tot.detach().cpu().numpy().view(np.uint8).tobytes()
    e, w = np.frombuffer(raw[:16], np.float64)
    pairs = int(np.frombuffer(raw[16:24], np.uint64)[0])
    return {"energy": float(e), "virial": float(w), "pairs": pairs}


def totals_from_array(tot) -> list:
    """Decodes k lj_totals held in a (k, 4) float64 tensor."""
    raw = np.ascontiguousarray(tot.detach().cpu().numpy()).view(np.uint8).reshape(-1, 32)
    out = []
    for r in raw:
        e, w = np.frombuffer(r[:16].tobytes(), np.float64)
        out.append({"energy": float(e), "virial": float(w), "pairs": int(np.frombuffer(r[16:24].tobytes(),
                                                                                         np.uint64)[0])})
    return out


# ------------------------------------------------------------------ batched systems
class _Drand48:
    """POSIX drand48 stream (srand48 semantics) for host-side workload parameters."""

    def __init__(self, seed: int):
        self.x = ((seed & 0xFFFFFFFF) << 16) | 0x330E

    def __call__(self) -> float:
        self.x = (0x5DEECE66D * self.x + 0xB) & ((1 << 48) - 1)
        return self.x / float(1 << 48)


def batch_workload(nsys: int = 512, seed: int = 1234, n_min: int = 1000, n_max: int = 200_000,
                   nb_min: float = 20.0, nb_max: float = 200.0, shell_fraction: float = 0.25) -> list:
    """Uneven systems: N log-uniform in [n_min, n_max], a mean neighbour count
    uniform in [nb_min, nb_max] fixing each cutoff, a share of sphere-surface
    systems (unit sphere about (0.5, 0.5, 0.5), box [-0.5, 1.5]^3) assigned by
    a seeded shuffle, the rest uniform in [0, 1)^3; sigma = cutoff / 2.5.
    Parameters come from one drand48 stream seeded with `seed`; system s's
    positions use seed + s."""
    d = _Drand48(seed)
    nshell = int(round(nsys * shell_fraction))
    kinds = ["shell"] * nshell + ["uniform"] * (nsys - nshell)
    for i in range(nsys - 1, 0, -1):  # Fisher-Yates
        j = int(d() * (i + 1))
        kinds[i], kinds[j] = kinds[j], kinds[i]
    out = []
    ln = np.log(n_max / n_min)
    for s in range(nsys):
        n = int(round(np.exp(d() * ln) * n_min))
        nb = nb_min + (nb_max - nb_min) * d()
        if kinds[s] == "uniform":
            rc = float(np.float32((3.0 * nb / (4.0 * np.pi * n)) ** (1.0 / 3.0)))
            lo, hi = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
        else:
            rc = float(np.float32(2.0 * np.sqrt(nb / n)))
            lo, hi = (-0.5, -0.5, -0.5), (1.5, 1.5, 1.5)
        out.append({"kind": kinds[s], "n": n, "cutoff": rc, "lo": lo, "hi": hi, "seed": seed + s,
                    "neighbours": nb})
    return out


class Batch:
    """An lj_batch: many systems, back to back in one SoA array, run as one step."""

    def __init__(self, ctx: Context, systems: list, cell_multiple: float = 1.0, threads: int = 128,
                 per_thread: int = 1):
        self.ctx = ctx
        self.systems = systems
        arr = (System * len(systems))()
        first = 0
        for s, d in enumerate(systems):
            a = arr[s]
            a.lo[:] = [float(v) for v in d["lo"]]
            a.hi[:] = [float(v) for v in d["hi"]]
            a.params = params(d["cutoff"], d.get("epsilon", 1.0), d.get("sigma"))
            a.first = first
            a.n = int(d["n"])
            d["first"] = first
            first += a.n
        self.ntotal = first
        cfg = BatchConfig(cell_multiple, threads, per_thread)
        h = C.c_void_p()
        _check(_lib.lj_batch_create(ctx.handle, len(systems), arr, C.byref(cfg), C.byref(h)), "lj_batch_create")
        self._h = h
        self._arr = arr

    def close(self):
        if getattr(self, "_h", None):
            _lib.lj_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def config(self) -> dict:
        c = BatchConfig()
        _check(_lib.lj_batch_get_config(self._h, C.byref(c)), "lj_batch_get_config")
        return {"cell_multiple": c.cell_multiple, "threads": c.threads, "per_thread": c.per_thread}

    def grid(self, s: int) -> Grid:
        g = Grid()
        _check(_lib.lj_batch_grid(self._h, s, C.byref(g)), "lj_batch_grid")
        return g

    def params(self, s: int) -> Params:
        return self._arr[s].params

    def generate(self):
        """Device positions of every system (seeded drand48), back to back."""
        t = self.ctx.torch
        x, y, z = (t.empty(max(self.ntotal, 1), dtype=t.float32, device=self.ctx.device) for _ in range(3))
        for d in self.systems:
            f, n = d["first"], d["n"]
            if n == 0:
                continue
            p = Particles(x.data_ptr() + 4 * f, y.data_ptr() + 4 * f, z.data_ptr() + 4 * f, None, None, n)
            if d["kind"] == "uniform":
                _check(_lib.lj_generate_uniform(self.ctx.handle, d["seed"], n, _f3(d["lo"]), _f3(d["hi"]),
                                                C.byref(p), None), "lj_generate_uniform")
            else:
                _check(_lib.lj_generate_sphere(self.ctx.handle, d["seed"], n, _f3((0.5, 0.5, 0.5)), 1.0,
                                               C.byref(p), None), "lj_generate_sphere")
        return x, y, z

    def alloc_outputs(self):
        t = self.ctx.torch
        n = max(self.ntotal, 1)
        dev = self.ctx.device
        return (t.empty(n, dtype=t.float32, device=dev), t.empty((n, 3), dtype=t.float32, device=dev),
                t.empty(n, dtype=t.int32, device=dev), t.zeros((len(self.systems), 4), dtype=t.float64, device=dev))

    def run(self, x, y, z, energy=None, force=None, index=None, totals=None, mode: str = "plain"):
        fn = {"plain": _lib.lj_batch_run, "graph": _lib.lj_batch_run_graph,
              "separate": _lib.lj_batch_run_separate}[mode]
        _check(fn(self.ctx.handle, self._h, _ptr(x), _ptr(y), _ptr(z), _ptr(energy), _ptr(force), _ptr(index),
                  _ptr(totals)), f"lj_batch_run ({mode})")

    def autotune(self, x, y, z):
        c = BatchConfig()
        ms = C.c_float(0)
        _check(_lib.lj_batch_autotune(self.ctx.handle, self._h, _ptr(x), _ptr(y), _ptr(z), C.byref(c),
                                      C.byref(ms)), "lj_batch_autotune")
        return {"cell_multiple": c.cell_multiple, "threads": c.threads, "per_thread": c.per_thread}, float(ms.value)
