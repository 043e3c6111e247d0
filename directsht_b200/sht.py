"""Drop-in ``DirectSHT`` backed by the sm_100a kernels of libdsht_b200.so.

Mirrors the reference's ``sht/sht.py:30-283`` interface: the constructor arguments,
``indx``, ``get_Ylm``/``get_dYlm``, ``alm2cl``, ``__call__`` and ``basic_sht``, with the
same Healpy alm ordering, return types and exceptions.  Inputs may be numpy arrays
(results come back as numpy) or CUDA torch tensors (results stay on the device).
PyTorch supplies device memory and the current stream; all arithmetic runs in the
library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as ct
import time

import numpy as np
import torch

from . import _lib as L


def _as_device_f64(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float64).contiguous()
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return torch.from_numpy(arr).to(device=device, non_blocking=False)


class DirectSHT:
    """Brute-force spherical harmonic transforms on a B200 (``sht/sht.py:30``)."""

    def __init__(self, Nell, Nx, xmax=0.75, dflt_type="float64", null_unphysical=True, device=None,
                 precision="fp64", compact_tables=False, table_layout="healpix", f32_tables=None):
        """Build the FP64 Ylm/dYlm tables on the GPU (``sht/sht.py:32-56``).

        :param Nell: number of ells (and m's).
        :param Nx: number of x = |cos theta| grid points in [0, xmax].
        :param xmax: largest |cos theta| handled without rotation.
        :param dflt_type: dtype of the host copy of the x grid (the tables are FP64).
        :param null_unphysical: accepted for compatibility; rows l < m are never stored, and
            the JAX layout's unphysical entries (l >= Nell) always read as zero.
        :param device: CUDA device (default: the current one).
        :param precision: "fp64" (agrees with the reference to ~1e-15), "mixed" (tensor-core
            per-bin sums and a tensor-core contraction of 4-byte fixed-point copies of the
            tables: fastest, <= 1e-7 x max|alm|) or "mixed_f64_tables" (tensor-core sums, FP64
            tables through the CUDA-core contraction).
        :param compact_tables: keep only the 4-byte fixed-point tables (half the memory of the
            FP64 pair; the plan then runs at precision "mixed" only, and get_Ylm/get_dYlm return
            the stored values, within 2^-31 of each row's largest entry).
        :param f32_tables: former name of ``compact_tables``.
        :param table_layout: layout of the host attributes ``Yv``/``Yd``: "healpix" (Nlm, Nx) rows
            in Healpy order, as the reference's numpy path stores them, or "jax" (Nell, Nell, Nx)
            indexed [m, ell - m, :], as its JAX path stores them (``sht/legendre_jax.py:14-25``).
        """
        if f32_tables is not None:
            compact_tables = f32_tables
        if table_layout not in ("healpix", "jax"):
            raise ValueError(f"table_layout must be 'healpix' or 'jax', not {table_layout!r}")
        self.table_layout = table_layout
        self._lib = L.load()
        if not torch.cuda.is_available():
            raise RuntimeError("DirectSHT (directsht_b200) needs a CUDA device; there is no CPU fallback")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self.Nell, self.Nx, self.xmax = int(Nell), int(Nx), float(xmax)
        self.Nlm = (self.Nell * (self.Nell + 1)) // 2
        xx = np.arange(Nx, dtype=dflt_type)
        xx *= xmax / float(Nx - 1)
        self.x = xx
        self._plan = ct.c_void_p()
        with torch.cuda.device(self.device):
            flags = L.DSHT_PLAN_F32_TABLES if compact_tables else L.DSHT_PLAN_DEFAULT
            L.check(self._lib.dsht_plan_create(self.Nell, self.Nx, self.xmax, flags, ct.byref(self._plan)))
        self.precision = None
        self._f32_only = bool(compact_tables)
        self.set_precision("mixed" if compact_tables else precision)
        self._Yv = None
        self._Yd = None
        self.verbose_timing = None

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                with torch.cuda.device(self.device):
                    self._lib.dsht_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def set_precision(self, precision):
        """Switch between "fp64", "mixed" and "mixed_f64_tables" (see the constructor)."""
        code = {"fp64": L.DSHT_PREC_FP64, "mixed": L.DSHT_PREC_MIXED,
                "mixed_f64_tables": L.DSHT_PREC_MIXED_F64_TABLES}.get(precision)
        if code is None:
            raise ValueError(f"precision must be 'fp64', 'mixed' or 'mixed_f64_tables', not {precision!r}")
        L.check(self._lib.dsht_set_precision(self._plan, code))
        self.precision = precision

    # -- tables ---------------------------------------------------------------------
    _BIN_SUMS = {"auto": L.DSHT_BIN_SUMS_AUTO, "nufft": L.DSHT_BIN_SUMS_NUFFT, "tc": L.DSHT_BIN_SUMS_TC,
                 "fp64": L.DSHT_BIN_SUMS_FP64}

    def tune(self, piece_max=None, maps_per_pass=None, bin_sums=None):
        """Set tuning parameters (``dsht_plan_tune``); None leaves one unchanged, 0 (or
        'auto') restores the automatic choice.  bin_sums picks the mixed levels' per-bin sums:
        'nufft', 'tc' (direct tensor-core sums), 'fp64' (direct FP64 sums) or 'auto' (the
        default).  Returns the current values
        as a dict (bin_sums as its name)."""
        if piece_max is not None:
            L.check(self._lib.dsht_plan_tune(self._plan, L.DSHT_TUNE_PIECE_MAX, int(piece_max)))
        if maps_per_pass is not None:
            L.check(self._lib.dsht_plan_tune(self._plan, L.DSHT_TUNE_MAPS_PER_PASS, int(maps_per_pass)))
        if bin_sums is not None:
            code = self._BIN_SUMS[bin_sums] if isinstance(bin_sums, str) else int(bin_sums)
            L.check(self._lib.dsht_plan_tune(self._plan, L.DSHT_TUNE_BIN_SUMS, code))
        out = {}
        for name, code in (("piece_max", L.DSHT_TUNE_PIECE_MAX), ("maps_per_pass", L.DSHT_TUNE_MAPS_PER_PASS),
                           ("bin_sums", L.DSHT_TUNE_BIN_SUMS)):
            v = ct.c_int()
            L.check(self._lib.dsht_plan_get_tune(self._plan, code, ct.byref(v)))
            out[name] = v.value
        out["bin_sums"] = {v: k for k, v in self._BIN_SUMS.items()}[out["bin_sums"]]
        return out

    def indx(self, ell, m):
        """Healpy index (``sht/sht.py:58-67``)."""
        return (m * (2 * self.Nell - 1 - m)) // 2 + ell

    def _row(self, which, ell, m):
        out = np.empty(self.Nx, dtype=np.float64)
        with torch.cuda.device(self.device):
            L.check(self._lib.dsht_get_row(self._plan, which, int(ell), int(m), L.dptr(out)))
        return out

    def get_Ylm(self, ell, m):
        """Ylm(x_i, 0) on the grid (``sht/sht.py:69-80``)."""
        return self._row(0, ell, m)

    def get_dYlm(self, ell, m):
        """d/dx Ylm(x_i, 0) on the grid (``sht/sht.py:82-93``)."""
        return self._row(1, ell, m)

    def _table(self, which):
        if self.table_layout == "jax":
            out = np.empty((self.Nell, self.Nell, self.Nx), dtype=np.float64)
            with torch.cuda.device(self.device):
                L.check(self._lib.dsht_get_table_mlayout(self._plan, which, L.ptr(out), 0, None))
            return out
        out = np.empty((self.Nlm, self.Nx), dtype=np.float64)
        with torch.cuda.device(self.device):
            L.check(self._lib.dsht_get_table(self._plan, which, L.dptr(out)))
        return out

    def table_on_device(self, which="Yv"):
        """A float64 CUDA tensor (Nell, Nell, Nx) of a table (``which`` = "Yv" or "Yd") in the
        JAX path's layout [m, ell - m, :] (``sht/legendre_jax.py:14-25``), zero where ell >=
        Nell, made on the device without passing through host memory."""
        code = {"Yv": 0, "Yd": 1}[which]
        out = torch.empty((self.Nell, self.Nell, self.Nx), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            L.check(self._lib.dsht_get_table_mlayout(self._plan, code, L.ptr(out), 1, ct.c_void_p(stream)))
        return out

    @property
    def Yv(self):
        """Host copy of the Ylm table (made on first use): (Nlm, Nx) in Healpy row order, or
        (Nell, Nell, Nx) indexed [m, ell - m] with table_layout="jax"."""
        if self._Yv is None:
            self._Yv = self._table(0)
        return self._Yv

    @property
    def Yd(self):
        """Host copy of the dYlm/dx table (made on first use)."""
        if self._Yd is None:
            self._Yd = self._table(1)
        return self._Yd

    def alm2cl(self, alm):
        """1/(2l+1) sum_m |alm|^2 (``sht/sht.py:95-109``).

        A numpy alm gives a numpy spectrum (computed on the host).  A CUDA tensor of complex128
        alm, shape (Nlm,) or (nmaps, Nlm), is reduced on its device without a copy to the host
        and gives a CUDA float64 tensor of shape (Nell,) or (nmaps, Nell)."""
        if isinstance(alm, torch.Tensor) and alm.is_cuda:
            a = alm.detach()
            if a.dtype != torch.complex128:
                a = a.to(torch.complex128)
            squeeze = a.dim() == 1
            a = a.reshape(-1, a.shape[-1])
            if a.shape[-1] != self.Nlm:
                raise ValueError(f"alm has {a.shape[-1]} entries per map, expected Nlm={self.Nlm}")
            a = a.contiguous()
            cl = torch.empty((a.shape[0], self.Nell), dtype=torch.float64, device=a.device)
            with torch.cuda.device(a.device):
                stream = torch.cuda.current_stream(a.device).cuda_stream
                L.check(self._lib.dsht_alm2cl_device(self.Nell, a.shape[0], L.ptr(a), 2 * self.Nlm, L.ptr(cl),
                                                     ct.c_void_p(stream)))
            return cl[0] if squeeze else cl
        if isinstance(alm, torch.Tensor):
            alm = alm.detach().numpy()
        a = np.ascontiguousarray(np.asarray(alm, dtype=np.complex128))
        cl = np.zeros(self.Nell)
        L.check(self._lib.dsht_alm2cl(self.Nell, a.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double)),
                                      L.dptr(cl)))
        return cl

    # -- transforms -----------------------------------------------------------------
    def _execute(self, t, p, w, mode):
        on_device = isinstance(t, torch.Tensor) and t.is_cuda
        n = len(t)
        with torch.cuda.device(self.device):
            td = _as_device_f64(t, self.device)
            pd = _as_device_f64(p, self.device)
            wd = _as_device_f64(w, self.device)
            alm = torch.empty(self.Nlm, dtype=torch.complex128, device=self.device)
            nbytes = ct.c_size_t()
            L.check(self._lib.dsht_workspace_size(self._plan, n, ct.byref(nbytes)))
            ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = self._lib.dsht_execute(self._plan, L.ptr(td), L.ptr(pd), L.ptr(wd), n, mode, L.ptr(alm),
                                        L.ptr(ws), ws.numel(), ct.c_void_p(stream))
        return rc, (alm if on_device else alm.cpu().numpy())

    def __call__(self, t, p, w):
        """alm of weighted points at (theta, phi) (``sht/sht.py:112-150``).

        Points with |cos theta| >= xmax are rotated by 90 degrees, transformed and
        their alm rotated back, all on the GPU.  Returns complex128 alm in Healpy order.
        """
        if not (len(t) == len(p) and len(p) == len(w)):
            raise AssertionError("theta,phi,wt must be the same length.")
        rc, alm = self._execute(t, p, w, L.DSHT_MODE_CALL)
        if rc == L.DSHT_ERR_POLAR_RANGE:
            # sht/sht.py:141-148: the polar transform failed; the reference prints and
            # returns the (still zero) alm without the equatorial part.
            print(f"AssertionError in basic_sht: theta must be in [ACos[xmax],ACos[-xmax]).")
            if self.xmax < np.sin(np.pi / 4):
                print("Warning: xmax is smaller than sin(pi/4), so some points may"
                      " still lie in the polar cap after rotation by 90 degrees."
                      " Trying increasing it.")
            return alm * 0
        if rc == L.DSHT_ERR_THETA_RANGE:
            raise AssertionError("theta must be in [ACos[xmax],ACos[-xmax]).")
        L.check(rc)
        return alm

    def call_maps(self, t, p, wts, mode="call"):
        """alm of several weight maps on one point set: row k is ``self(t, p, wts[k])``
        (or ``self.basic_sht(t, p, wts[k])`` with mode="basic").

        The reference has no multi-map call; its users loop ``__call__``
        (``sht/sht.py:112-150``) over the maps.  ``wts`` has shape (nmaps, N), float64 or
        float32 (float32 weights are used exactly, without a float64 copy).  The points
        are classified and sorted once.  Returns complex128 alm of shape (nmaps, Nlm).
        """
        on_device = isinstance(t, torch.Tensor) and t.is_cuda
        n = len(t)
        if isinstance(wts, torch.Tensor):
            wd = wts.to(device=self.device)
        else:
            wd = torch.from_numpy(np.ascontiguousarray(np.asarray(wts)))
        if wd.dim() == 1:
            wd = wd[None, :]
        if wd.dtype not in (torch.float32, torch.float64):
            wd = wd.to(torch.float64)
        if not (len(t) == len(p) and wd.shape[1] == len(p)):
            raise AssertionError("theta,phi,wt must be the same length.")
        nmaps = int(wd.shape[0])
        dtype = L.DSHT_W_F32 if wd.dtype == torch.float32 else L.DSHT_W_F64
        with torch.cuda.device(self.device):
            td = _as_device_f64(t, self.device)
            pd = _as_device_f64(p, self.device)
            wd = wd.to(device=self.device).contiguous()
            alm = torch.empty((nmaps, self.Nlm), dtype=torch.complex128, device=self.device)
            nbytes = ct.c_size_t()
            L.check(self._lib.dsht_workspace_size_maps(self._plan, n, nmaps, ct.byref(nbytes)))
            ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            code = L.DSHT_MODE_CALL if mode == "call" else L.DSHT_MODE_BASIC
            rc = self._lib.dsht_execute_maps(self._plan, L.ptr(td), L.ptr(pd), L.ptr(wd), dtype, n, nmaps,
                                             wd.stride(0), code, L.ptr(alm), L.ptr(ws), ws.numel(),
                                             ct.c_void_p(stream))
        if rc == L.DSHT_ERR_POLAR_RANGE:
            print(f"AssertionError in basic_sht: theta must be in [ACos[xmax],ACos[-xmax]).")
            alm.zero_()
        elif rc == L.DSHT_ERR_THETA_RANGE:
            raise AssertionError("theta must be in [ACos[xmax],ACos[-xmax]).")
        elif rc == L.DSHT_ERR_EMPTY:
            raise ValueError("The theta array seems to be empty!")
        else:
            L.check(rc)
        return alm if on_device else alm.cpu().numpy()

    def call_batch(self, point_sets, mode="call"):
        """alm of several independent point sets, each ``(theta, phi, w)``: item i is
        ``self(*point_sets[i])`` (or ``basic_sht`` with mode="basic").

        The reference has no batch call; its users loop ``__call__`` (``sht/sht.py:112-150``).
        Here the contraction of up to four point sets shares one read of the tables and the
        rotation of up to eight shares one Wigner-d recursion.  Returns a list of complex128
        alm (numpy, or CUDA tensors when the inputs are CUDA tensors).  A transform whose polar
        points cannot be rotated into range gives zeros, as ``__call__`` does.
        """
        code = L.DSHT_MODE_CALL if mode == "call" else L.DSHT_MODE_BASIC
        n = len(point_sets)
        if n == 0:
            return []
        on_device = isinstance(point_sets[0][0], torch.Tensor) and point_sets[0][0].is_cuda
        with torch.cuda.device(self.device):
            dev = []
            for t, p, w in point_sets:
                if not (len(t) == len(p) and len(p) == len(w)):
                    raise AssertionError("theta,phi,wt must be the same length.")
                dev.append(tuple(_as_device_f64(a, self.device) for a in (t, p, w)))
            alms = [torch.empty(self.Nlm, dtype=torch.complex128, device=self.device) for _ in range(n)]
            Ns = (ct.c_int64 * n)(*[len(d[0]) for d in dev])
            arr = lambda xs: (ct.c_void_p * n)(*[x.data_ptr() for x in xs])
            status = torch.zeros(n, dtype=torch.int32, device=self.device)
            nbytes = ct.c_size_t()
            L.check(self._lib.dsht_workspace_size_batch(self._plan, max(Ns), n, ct.byref(nbytes)))
            ws = torch.empty(max(int(nbytes.value), 1), dtype=torch.uint8, device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            rc = self._lib.dsht_enqueue_batch(self._plan, n, arr([d[0] for d in dev]), arr([d[1] for d in dev]),
                                              arr([d[2] for d in dev]), Ns, code, arr(alms), L.ptr(status),
                                              L.ptr(ws), ws.numel(), ct.c_void_p(stream))
            if rc == L.DSHT_ERR_EMPTY:
                raise ValueError("The theta array seems to be empty!")
            L.check(rc)
            flags = status.cpu().numpy().astype(np.uint32)
        for i, f in enumerate(flags):
            rc = self._lib.dsht_status(int(f), code)
            if rc == L.DSHT_ERR_POLAR_RANGE and code == L.DSHT_MODE_CALL:
                print(f"AssertionError in basic_sht: theta must be in [ACos[xmax],ACos[-xmax]).")
                alms[i].zero_()
            elif rc == L.DSHT_ERR_THETA_RANGE:
                raise AssertionError("theta must be in [ACos[xmax],ACos[-xmax]).")
            else:
                L.check(rc)
        return alms if on_device else [a.cpu().numpy() for a in alms]

    def basic_sht(self, theta, phi, wt, reg_factor=1.0, verbose=True):
        """alm of points with |cos theta| < xmax, no rotation (``sht/sht.py:153-283``).

        Like the reference, multiplies ``wt`` in place by ``reg_factor`` and divides the
        result by it.
        """
        if not (len(theta) == len(phi) and len(phi) == len(wt)):
            raise AssertionError("theta,phi,wt must be the same length.")
        t0 = time.time()
        wt *= reg_factor
        rc, alm = self._execute(theta, phi, wt, L.DSHT_MODE_BASIC)
        if rc == L.DSHT_ERR_THETA_RANGE:
            raise AssertionError("theta must be in [ACos[xmax],ACos[-xmax]).")
        if rc == L.DSHT_ERR_EMPTY:
            raise ValueError("The theta array seems to be empty!")
        L.check(rc)
        if verbose:
            print(f"basic_sht on the GPU took {time.time() - t0} seconds.", flush=True)
        return alm / reg_factor
