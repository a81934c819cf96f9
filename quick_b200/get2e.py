"""Host-side interface of the B200 get2e library.

Two faces, both thin layers over ``libquick_b200.so`` (``include/quick_b200.h``):

* :class:`Get2e` -- the context API: one molecule + basis resident on a GPU,
  Schwarz bounds computed on the device, Fock builds on device tensors
  (``fock2e``) or host arrays (``fock2e_host``).
* ``gpu_*`` functions -- the reference's Fortran-to-C call sequence
  (``src/modules/quick_scf_operator_module.f90:87-127``, ``src/main.f90:152-203``)
  with the same names, argument order and meaning, passing every argument by
  reference exactly as gfortran does, so tests read like QUICK's own driver.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from ._native import QuickError, check, lib

_c_int = ctypes.c_int
_c_double = ctypes.c_double
_c_bool = ctypes.c_bool


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def _i32(a):
    return np.asfortranarray(a, dtype=np.int32)


class Get2e:
    """One molecule's closed-shell two-electron Fock build on one GPU."""

    def __init__(self, basis, device: int = 0, integral_cutoff: float = 1e-7,
                 prim_limit: float = 1e-8, schwarz=None):
        L = lib()
        st = _c_int(0)
        self.h = L.qk_create(int(device), ctypes.byref(st))
        if not self.h:
            raise QuickError(st.value, "qk_create")
        self.device = device
        self.bind(basis, schwarz)
        self.set_cutoffs(integral_cutoff, prim_limit)

    def bind(self, basis, schwarz=None):
        """Put another molecule (or geometry) on this context: the device buffers
        are kept and grown as needed; Schwarz bounds are recomputed unless given."""
        L = lib()
        self.basis = basis
        b = basis
        self._keep = [np.ascontiguousarray(b.xyz, dtype=np.float64), _i32(b.kstart), _i32(b.katom),
                      _i32(b.kprim), _i32(b.ksumtype), _i32(b.qstart), _i32(b.qfinal),
                      _i32(b.qsbasis), _i32(b.qfbasis), _f64(b.gccoeff), _f64(b.cons),
                      _f64(b.gcexpo), _i32(b.klmn)]
        k = self._keep
        check(L.qk_set_basis(self.h, b.mol.natom, _p(k[0]), b.nshell, b.nbasis, b.jbasis,
                             *[_p(x) for x in k[1:]], int(b.gccoeff.shape[0])), "qk_set_basis")
        if schwarz is None:
            self.Ycut, self.cutprim = self.schwarz()
        else:
            self.set_schwarz(*schwarz)

    def close(self):
        if getattr(self, "h", None):
            lib().qk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- per-geometry set-up
    def schwarz(self):
        """Ycutoff (nshell^2) and cutprim (jbasis^2) computed on the GPU."""
        b = self.basis
        Y = np.zeros((b.nshell, b.nshell), order="F")
        cp = np.zeros((b.jbasis, b.jbasis), order="F")
        check(lib().qk_schwarz(self.h, _p(Y), _p(cp)), "qk_schwarz")
        return Y, cp

    def set_schwarz(self, Y, cutprim):
        self.Ycut, self.cutprim = _f64(Y), _f64(cutprim)
        check(lib().qk_set_schwarz(self.h, _p(self.Ycut), _p(self.cutprim)), "qk_set_schwarz")

    def set_precision(self, fp32_bound: float):
        """Mixed form: FP32 vertical recursion for quartets with Y_ij*Y_kl < fp32_bound
        (0 = plain FP64)."""
        self.fp32_bound = float(fp32_bound)
        check(lib().qk_set_precision(self.h, self.fp32_bound), "qk_set_precision")

    def set_boys(self, mode: int):
        """Boys function of the integrals: 0 = accurate (default); QUICK's own
        fmt.f90 formulas at the order its CPU get2e uses (1) or its GPU get2e uses
        (2), to reproduce the reference's numbers to the last digits."""
        check(lib().qk_set_boys(self.h, int(mode)), "qk_set_boys")

    def fp32_quartets(self):
        q = ctypes.c_longlong(0)
        check(lib().qk_last_work_mixed(self.h, ctypes.byref(q)), "qk_last_work_mixed")
        return q.value

    def set_cutoffs(self, integral_cutoff: float, prim_limit: float):
        self.integral_cutoff, self.prim_limit = float(integral_cutoff), float(prim_limit)
        check(lib().qk_set_cutoffs(self.h, self.integral_cutoff, self.prim_limit), "qk_set_cutoffs")

    # -- Fock builds
    def fock2e(self, D, o=None, cutmat=None, stream=None):
        """o += G(D) on the device; D, o, cutmat are CUDA float64 torch tensors.

        Returns o (allocated as zeros when not given).  Enqueued on ``stream``
        (default: torch's current stream); no synchronisation."""
        import torch
        n = self.basis.nbasis
        if D.dtype != torch.float64 or not D.is_cuda or tuple(D.shape) != (n, n):
            raise ValueError("D must be a CUDA float64 tensor of shape (nbasis, nbasis)")
        D = D.contiguous()
        if o is None:
            o = torch.zeros((n, n), dtype=torch.float64, device=D.device)
        if stream is None:
            stream = torch.cuda.current_stream(D.device)
        cm = ctypes.c_void_p(cutmat.data_ptr()) if cutmat is not None else None
        check(lib().qk_fock2e_device(self.h, ctypes.c_void_p(D.data_ptr()), cm,
                                     ctypes.c_void_p(o.data_ptr()), ctypes.c_void_p(stream.cuda_stream)),
              "qk_fock2e_device")
        return o

    def density_cutoff(self, D, out=None, stream=None):
        import torch
        ns = self.basis.nshell
        if out is None:
            out = torch.empty((ns, ns), dtype=torch.float64, device=D.device)
        if stream is None:
            stream = torch.cuda.current_stream(D.device)
        check(lib().qk_density_cutoff_device(self.h, ctypes.c_void_p(D.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()),
                                             ctypes.c_void_p(stream.cuda_stream)), "qk_density_cutoff_device")
        return out

    def fock2e_uhf(self, Da, Db, oa=None, ob=None, cutmat=None, stream=None):
        """Open-shell build: oa += G_alpha(Da, Db), ob += G_beta(Da, Db) on the device
        (CUDA float64 tensors); returns (oa, ob).  ``cutmat``: the open-shell density
        screen, or None to derive it from Da and Db."""
        import torch
        n = self.basis.nbasis
        for X in (Da, Db):
            if X.dtype != torch.float64 or not X.is_cuda or tuple(X.shape) != (n, n):
                raise ValueError("Da and Db must be CUDA float64 tensors of shape (nbasis, nbasis)")
        Da, Db = Da.contiguous(), Db.contiguous()
        oa = torch.zeros_like(Da) if oa is None else oa
        ob = torch.zeros_like(Db) if ob is None else ob
        if stream is None:
            stream = torch.cuda.current_stream(Da.device)
        cm = ctypes.c_void_p(cutmat.data_ptr()) if cutmat is not None else None
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        check(lib().qk_fock2e_uhf_device(self.h, vp(Da), vp(Db), cm, vp(oa), vp(ob),
                                         ctypes.c_void_p(stream.cuda_stream)), "qk_fock2e_uhf_device")
        return oa, ob

    def fock2e_host(self, D, o=None, cutmat=None):
        """Host arrays: returns o + G(D) (copies in, computes, copies out)."""
        n = self.basis.nbasis
        D = np.ascontiguousarray(D, dtype=np.float64)
        out = np.zeros((n, n)) if o is None else np.array(o, dtype=np.float64, order="C", copy=True)
        cm = _p(np.ascontiguousarray(cutmat, dtype=np.float64)) if cutmat is not None else None
        if cutmat is not None:
            cm_arr = np.ascontiguousarray(cutmat, dtype=np.float64)
            cm = _p(cm_arr)
        check(lib().qk_fock2e_host(self.h, _p(D), cm, _p(out)), "qk_fock2e_host")
        return out

    # -- sharded builds (one molecule over several GPUs)
    def set_shard(self, rank: int, count: int):
        """Keep every ``count``-th work item of each class, starting at ``rank``
        ((0, 1) = all); the work lists are rebuilt at the next build."""
        check(lib().qk_set_shard(self.h, int(rank), int(count)), "qk_set_shard")

    def accumulate(self, D, A, cutmat=None, stream=None):
        """This context's share of G(D) added into ``A``: an int64 (nbasis, nbasis)
        CUDA tensor of fixed-point sums (2^-44 units) that the caller clears."""
        import torch
        n = self.basis.nbasis
        if D.shape != (n, n) or A.shape != (n, n) or A.dtype != torch.int64 or not A.is_contiguous():
            raise ValueError("accumulate: D must be (n, n) float64 and A a contiguous (n, n) int64 tensor")
        D = D.contiguous()
        s = stream if stream is not None else torch.cuda.current_stream(D.device)
        cm = ctypes.c_void_p(cutmat.data_ptr()) if cutmat is not None else None
        check(lib().qk_fock2e_device_accumulate(self.h, ctypes.c_void_p(D.data_ptr()), cm,
                                                ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(s.cuda_stream)),
              "qk_fock2e_device_accumulate")
        return A

    def fock2e_sharded(self, D, o=None, group=None):
        """o += G(D) with the work split over the ranks of ``group`` (torch.distributed,
        one rank per GPU): each rank builds its share into an int64 accumulator, one
        integer all-reduce sums them (exact, so the result equals the one-GPU build bit
        for bit), and every rank finalises the same o.  Call ``set_shard(rank, size)``
        first (``shard_for``)."""
        import torch
        n = self.basis.nbasis
        if o is None:
            o = torch.zeros((n, n), dtype=torch.float64, device=D.device)
        A = torch.zeros((n, n), dtype=torch.int64, device=D.device)
        self.accumulate(D, A)
        allreduce_fixed(A, group)
        s = torch.cuda.current_stream(D.device)
        check(lib().qk_finalize_fixed(ctypes.c_void_p(A.data_ptr()), n, ctypes.c_void_p(o.data_ptr()),
                                      ctypes.c_void_p(s.cuda_stream)), "qk_finalize_fixed")
        return o

    def shard_for(self, group=None):
        """set_shard(rank, world size) of ``group``."""
        import torch.distributed as dist
        self.set_shard(dist.get_rank(group), dist.get_world_size(group))

    def set_worklist_builder(self, on_device: bool):
        """Build the work lists on the GPU (default) or on the host (same lists)."""
        check(lib().qk_set_worklist_builder(self.h, int(bool(on_device))), "qk_set_worklist_builder")

    def set_merge_sp(self, on: bool):
        """The s/p classes as one persistent kernel per precision (qk_set_merge_sp)."""
        check(lib().qk_set_merge_sp(self.h, 1 if on else 0), "qk_set_merge_sp")

    def set_streams(self, nstreams: int):
        """Class kernels over ``nstreams`` concurrent streams (0: one after another)."""
        check(lib().qk_set_streams(self.h, int(nstreams)), "qk_set_streams")

    def prepare(self):
        """Build the pair tables and work lists now rather than in the first build."""
        check(lib().qk_prepare(self.h), "qk_prepare")

    def device_bytes(self):
        """(total, work-list) bytes of device memory held by the context."""
        t = ctypes.c_ulonglong(0)
        it = ctypes.c_ulonglong(0)
        check(lib().qk_device_bytes(self.h, ctypes.byref(t), ctypes.byref(it)), "qk_device_bytes")
        return t.value, it.value

    def work(self):
        q = ctypes.c_longlong(0)
        pq = ctypes.c_longlong(0)
        nl = ctypes.c_int(0)
        check(lib().qk_last_work(self.h, ctypes.byref(q), ctypes.byref(pq), ctypes.byref(nl)), "qk_last_work")
        return {"quartets": q.value, "prim_quartets": pq.value, "launches": nl.value}


class Get2eBatch:
    """Fock builds of many molecules at once on one GPU (``qk_batch_*``).

    Every molecule keeps its own :class:`Get2e` context (basis, Schwarz bounds,
    cutoffs, precision); one call builds ``o[m] += G(D[m])`` for all of them with
    one launch per integral class over the merged work lists, so that molecules
    too small to fill the GPU alone share it.  Results equal the one-molecule
    builds bit for bit (same quartets, same int64 accumulation)."""

    def __init__(self, device: int = 0):
        st = _c_int(0)
        self.h = lib().qk_batch_create(int(device), ctypes.byref(st))
        if not self.h:
            raise QuickError(st.value, "qk_batch_create")
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().qk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve_sms(self, sms: int):
        """Leave ``sms`` SMs free of the batch's class kernels (for concurrent work)."""
        check(lib().qk_batch_reserve_sms(self.h, int(sms)), "qk_batch_reserve_sms")

    def fock2e(self, engines, Ds, os=None, cutmats=None, stream=None):
        """o[m] += G(D[m]) for every engine m; tensors are CUDA float64.

        Returns the list of o tensors (zeros allocated where not given).
        Enqueued on ``stream`` (default: torch's current stream)."""
        import torch
        n = len(engines)
        if n == 0:
            return []
        if len(Ds) != n:
            raise ValueError("one density per engine")
        Ds = [D.contiguous() for D in Ds]
        if os is None:
            os = [None] * n
        os = list(os)
        for m, (e, D) in enumerate(zip(engines, Ds)):
            nb = e.basis.nbasis
            if D.dtype != torch.float64 or not D.is_cuda or tuple(D.shape) != (nb, nb):
                raise ValueError(f"D[{m}] must be a CUDA float64 tensor of shape ({nb}, {nb})")
            if os[m] is None:
                os[m] = torch.zeros((nb, nb), dtype=torch.float64, device=D.device)
        if stream is None:
            stream = torch.cuda.current_stream(Ds[0].device)
        VP = ctypes.c_void_p
        hs = (VP * n)(*[e.h for e in engines])
        dp = (VP * n)(*[D.data_ptr() for D in Ds])
        op = (VP * n)(*[o.data_ptr() for o in os])
        cp = None
        if cutmats is not None:
            cp = (VP * n)(*[c.data_ptr() if c is not None else None for c in cutmats])
        check(lib().qk_batch_fock2e(self.h, n, hs, dp, cp, op, VP(stream.cuda_stream)), "qk_batch_fock2e")
        return os


# ---------------------------------------------------------------------------
# The reference's Fortran -> C call sequence (all arguments by reference).
# ---------------------------------------------------------------------------
def allreduce_fixed(A, group=None):
    """Sum int64 fixed-point accumulators over the ranks of ``group`` in place (a
    no-op without an initialised process group).  Integer addition is exact and
    order-free, so every rank ends with the same bits whatever the reduction order
    (NCCL on GPUs, gloo on CPUs)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(A, op=dist.ReduceOp.SUM, group=group)
    return A


def _ref(x, ctype):
    return ctypes.byref(ctype(x))


def gpu_new():
    ierr = _c_int(0)
    lib().gpu_new_(ctypes.byref(ierr))
    return ierr.value


def gpu_init_device():
    ierr = _c_int(0)
    lib().gpu_init_device_(ctypes.byref(ierr))
    return ierr.value


def gpu_setup(natom, nbasis, nelec, imult, molchg, iattype):
    lib().gpu_setup_(_ref(natom, _c_int), _ref(nbasis, _c_int), _ref(nelec, _c_int),
                     _ref(imult, _c_int), _ref(molchg, _c_int), _ref(iattype, _c_int))


def gpu_upload_method(method=0, is_oshell=False, hyb_coeff=1.0):
    lib().gpu_upload_method_(_ref(method, _c_int), _ref(is_oshell, _c_bool), _ref(hyb_coeff, _c_double))


def gpu_upload_xyz(xyz):
    x = np.ascontiguousarray(xyz, dtype=np.float64)   # xyz(3, natom) column-major
    lib().gpu_upload_xyz_(_p(x))


def gpu_upload_basis(b):
    """gpu_upload_basis_ with QUICK's 29 arguments (src/gpu/cuda/gpu.cu:1782)."""
    z = np.zeros(max(b.mol.natom, b.nshell, 1), dtype=np.int32)
    args = [
        _ref(b.nshell, _c_int), _ref(b.nprim, _c_int), _ref(b.nshell, _c_int), _ref(b.jbasis, _c_int),
        _ref(b.maxcontract, _c_int), _i32(b.ncontract), _i32(b.itype), _f64(b.aexp), _f64(b.dcoeff),
        z, z, z, z, _i32(b.ncenter), _i32(b.kstart), _i32(b.katom), _i32(b.ktype), _i32(b.kprim),
        np.zeros(93, dtype=np.int32), _i32(b.ksumtype), _i32(b.qnumber), _i32(b.qstart),
        _i32(b.qfinal), _i32(b.qsbasis), _i32(b.qfbasis), _f64(b.gccoeff), _f64(b.cons),
        _f64(b.gcexpo), _i32(b.klmn)]
    keep = [a for a in args if isinstance(a, np.ndarray)]
    cargs = [_p(a) if isinstance(a, np.ndarray) else a for a in args]
    lib().gpu_upload_basis_(*cargs)
    del keep


def gpu_upload_cutoff_matrix(Ycutoff, cutprim):
    Y, cp = _f64(Ycutoff), _f64(cutprim)
    lib().gpu_upload_cutoff_matrix_(_p(Y), _p(cp))


def gpu_upload_calculated(o, co, vec, dense):
    o, co, vec, dense = _f64(o), _f64(co), _f64(vec), _f64(dense)
    lib().gpu_upload_calculated_(_p(o), _p(co), _p(vec), _p(dense))


def gpu_upload_cutoff(cutmatrix, integral_cutoff, prim_limit, dm_cutoff=1e-10, core_cutoff=1e-12):
    cm = _f64(cutmatrix)
    lib().gpu_upload_cutoff_(_p(cm), _ref(integral_cutoff, _c_double), _ref(prim_limit, _c_double),
                             _ref(dm_cutoff, _c_double), _ref(core_cutoff, _c_double))


def gpu_get_cshell_eri(deltaO, o):
    """o (Fortran-ordered float64 array) += G(dense); modified in place."""
    if not (isinstance(o, np.ndarray) and o.dtype == np.float64 and o.flags.f_contiguous):
        raise ValueError("o must be a Fortran-ordered float64 array")
    lib().gpu_get_cshell_eri_(_ref(bool(deltaO), _c_bool), _p(o))


def gpu_upload_calculated_beta(ob, denseb):
    ob, denseb = _f64(ob), _f64(denseb)
    lib().gpu_upload_calculated_beta_(_p(ob), _p(denseb))


def gpu_get_oshell_eri(deltaO, o, ob):
    """o += G_alpha, ob += G_beta (Fortran-ordered float64 arrays, modified in place)."""
    for a in (o, ob):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous):
            raise ValueError("o and ob must be Fortran-ordered float64 arrays")
    lib().gpu_get_oshell_eri_(_ref(bool(deltaO), _c_bool), _p(o), _p(ob))


def gpu_delete():
    ierr = _c_int(0)
    lib().gpu_delete_(ctypes.byref(ierr))
    return ierr.value


def last_status():
    return lib().qk_last_status()
