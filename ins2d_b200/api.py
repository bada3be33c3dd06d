"""Host-side mirror of the reference's hot-path interface over libins2d.so.

The reference (bsanderse/INS2D, MATLAB) exposes the path as functions of an
``options`` struct:

  [maxres,F,dF] = F(V,C,p,T,t,options,getJacobian,nopressure)   spatial/F.m:1
  dp = pressure_poisson(f,t,options)              solvers/pressure/pressure_poisson.m:1
  p  = pressure_additional_solve(V,p,T,t,options) solvers/pressure/pressure_additional_solve.m:1
  [Vnew,pnew,Tnew] = time_ERK(Vn,pn,Tn,tn,dt,options)  unsteady/time_ERK.m:1
  [maxdiv,umom,vmom,k] = check_conservation(V,T,t,options)  spatial/check_conservation.m:1

Here ``options`` is an :class:`Options` (a device context built from the
grid, the boundary-condition types, the case's uBC/vBC functions and the
solver settings), and module-level functions with the reference's names and
argument order call into it.  Arrays are numpy float64 vectors (host memory,
copied in and out) or contiguous float64 CUDA tensors (used in place), in the
reference's ordering (x fastest, V = [u; v]).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .rk import getRKmethod


class Ins2dError(RuntimeError):
    """Raised for a non-zero status of the C-ABI (the reference raises a
    MATLAB error in the same situations, e.g. cg.F:262)."""

    def __init__(self, status, msg):
        super().__init__(f"{_lib.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _zero_bc(x, y, t):
    return np.zeros(np.size(x) * np.size(y))


def _mesh_positions(x, y, BC):
    """xin / yin of operator_mesh.m:185-249, 272-320."""
    L, R = BC["u"]["left"], BC["u"]["right"]
    if L == "dir" and R == "dir":
        xin = x[1:-1]
    elif L == "dir" and R == "pres":
        xin = x[1:]
    elif L == "pres" and R == "dir":
        xin = x[:-1]
    elif L == "pres" and R == "pres":
        xin = x.copy()
    elif L == "per" and R == "per":
        xin = x[:-1]
    else:
        raise ValueError(f"unsupported u-left/u-right combination {L}/{R}")
    Lo, Up = BC["v"]["low"], BC["v"]["up"]
    if Lo == "dir" and Up == "dir":
        yin = y[1:-1]
    elif Lo == "dir" and Up == "pres":
        yin = y[1:]
    elif Lo == "pres" and Up == "dir":
        yin = y[:-1]
    elif Lo == "pres" and Up == "pres":
        yin = y.copy()
    elif Lo == "per" and Up == "per":
        yin = y[:-1]
    else:
        raise ValueError(f"unsupported v-low/v-up combination {Lo}/{Up}")
    return xin, yin


def _is_torch_cuda(a):
    return hasattr(a, "is_cuda") and hasattr(a, "data_ptr") and a.is_cuda


class _Arr:
    """A float64 array argument: host numpy (copied) or CUDA tensor (in place)."""

    def __init__(self, a, n, name):
        if _is_torch_cuda(a):
            import torch
            if a.dtype != torch.float64 or not a.is_contiguous() or a.numel() != n:
                raise ValueError(f"{name}: need a contiguous float64 CUDA tensor of {n} elements")
            self.dev = True
            self.obj = a
            self.ptr = a.data_ptr()
        else:
            arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
            if arr.size != n:
                raise ValueError(f"{name}: expected {n} values, got {arr.size}")
            self.dev = False
            self.obj = arr
            self.ptr = arr.ctypes.data


class Options:
    """The ``options`` struct of the hot path, backed by a device context.

    Parameters mirror the reference's case parameters: grid-line coordinates
    ``x``, ``y`` (mesh_generation.m), boundary-condition types ``BC``
    (``{"u": {"left":..,"right":..,"low":..,"up":..}, "v": {...}}`` with
    'dir'/'pres'/'per'/'sym', boundary_conditions.m), the case's boundary
    functions ``uBC(x, y, t)`` / ``vBC`` (and ``dudtBC``/``dvdtBC`` for
    unsteady BCs), ``Re``, ``poisson`` (1-5: device PCG, 6: FFT), ``CG_acc``,
    ``CG_maxit``, ``p_add_solve``, the RK method name, ``precision``
    ('fp64' or 'fp32': FP32 convection/diffusion stencils) and ``precond``
    (PCG preconditioner: 'default' = fast diagonalization where it applies
    -- periodic uniform grids, or at most 1024 pressure cells per direction
    -- else multigrid where the grid allows it, else Jacobi; 'fdm', 'mg', or
    'jacobi').
    """

    def __init__(self, x, y, BC, Re=1000.0, poisson=4, CG_acc=1e-12, CG_maxit=10000, p_add_solve=1, RK="RK44",
                 uBC=None, vBC=None, dudtBC=None, dvdtBC=None, pLe=0.0, pRi=0.0, pLo=0.0, pUp=0.0,
                 precision="fp64", device=0, BC_unsteady=None, precond="default", _handle=None, **private):
        bad = [k for k in private if not k.startswith("_")]
        if bad:
            raise TypeError(f"unexpected options: {bad}")  # keys starting with '_' are annotations of a case
        self._lib = _lib.load()
        self._owner = _handle is None
        self._stream = None  # the cudaStream_t handle set by set_stream (None: the context's own)
        self.device = int(device)
        self.x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        self.y = np.ascontiguousarray(np.asarray(y, dtype=np.float64))
        self.BC = {"u": dict(BC["u"]), "v": dict(BC["v"])}
        unsteady = BC.get("BC_unsteady", 0) if BC_unsteady is None else BC_unsteady
        self.BC_unsteady = int(unsteady)
        self.Re = float(Re)
        self.poisson = int(poisson)
        self.uBC = uBC or _zero_bc
        self.vBC = vBC or _zero_bc
        self.dudtBC = dudtBC or _zero_bc
        self.dvdtBC = dvdtBC or _zero_bc
        self.pbc = (pLe, pRi, pLo, pUp)
        self.RK = RK
        self._ctx = ctypes.c_void_p()
        Nx, Ny = len(self.x) - 1, len(self.y) - 1
        g = _lib.GridDesc(Nx, Ny, self.x.ctypes.data_as(_lib.c_double_p), self.y.ctypes.data_as(_lib.c_double_p))
        codes = []
        for comp, sides in (("u", ("left", "right", "low", "up")), ("v", ("left", "right", "low", "up"))):
            for sd in sides:
                t = self.BC[comp][sd]
                if t not in _lib.BC_CODES:
                    raise ValueError(f"wrong BC for {comp}-{sd}: {t}")
                codes.append(_lib.BC_CODES[t])
        b = _lib.BcDesc(*codes, self.BC_unsteady)
        o = _lib.Opts()
        o.Re = self.Re
        o.poisson = self.poisson
        o.CG_acc = float(CG_acc)
        o.CG_maxit = int(CG_maxit)
        o.p_add_solve = int(p_add_solve)
        A, bb, c = getRKmethod(RK)
        s = len(bb)
        o.rk_stages = s
        for i in range(s):
            for j in range(s):
                o.rk_A[i * s + j] = A[i, j]
            o.rk_b[i] = bb[i]
            o.rk_c[i] = c[i]
        o.precision = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32_STENCIL}[precision]
        o.device = int(device)
        o.precond = _lib.PRECOND_CODES[precond]
        self._desc = (g, b, o)  # kept for ensembles
        if _handle is not None:
            self._ctx = ctypes.c_void_p(_handle)
        else:
            rc = self._lib.ins2d_ctx_create(ctypes.byref(g), ctypes.byref(b), ctypes.byref(o),
                                            ctypes.byref(self._ctx))
            if rc != 0:
                msg = self._err()
                self._lib.ins2d_ctx_destroy(self._ctx)
                self._ctx = None
                raise Ins2dError(rc, msg)
        sz = _lib.Sizes()
        self._lib.ins2d_get_sizes(self._ctx, ctypes.byref(sz))
        for f, _ in _lib.Sizes._fields_:
            setattr(self, f, int(getattr(sz, f)))
        self.xp = (self.x[:-1] + self.x[1:]) / 2
        self.yp = (self.y[:-1] + self.y[1:]) / 2
        self.xin, self.yin = _mesh_positions(self.x, self.y, self.BC)
        # positions of the unknowns (operator_mesh.m:401-409)
        self.xu = np.tile(self.xin, self.Nuy_in)
        self.yu = np.repeat(self.yp, self.Nux_in)
        self.xv = np.tile(self.xp, self.Nvy_in)
        self.yv = np.repeat(self.yin, self.Nvx_in)
        self._sampler = None
        if self.BC_unsteady and _handle is None:
            def _cb(user, t, ctx):
                try:
                    self.set_bc_vectors(t)
                    return 0
                except Exception:  # report through the C status
                    return _lib.EINVAL
            self._sampler = _lib.SAMPLER_FN(_cb)
            self._lib.ins2d_set_bc_sampler(self._ctx, self._sampler, None)
        if _handle is None:
            self.set_bc_vectors(0.0)

    # -- plumbing ------------------------------------------------------------
    def _err(self):
        m = self._lib.ins2d_last_error(self._ctx)
        return m.decode() if m else ""

    def _check(self, rc):
        if rc != 0:
            raise Ins2dError(rc, self._err())

    def close(self):
        if getattr(self, "_ctx", None):
            if getattr(self, "_owner", True):
                self._lib.ins2d_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _mem(self, *arrs):
        """MEM_HOST or MEM_DEVICE for the call's arrays; for device tensors the
        context's stream is first ordered after torch's current stream, so an
        input still being written by a torch kernel is read only when done."""
        kinds = {a.dev for a in arrs if a is not None}
        if len(kinds) > 1:
            raise ValueError("mix of host and device arrays")
        if kinds == {True}:
            _order_after_torch(self._lib.ins2d_wait_stream, self._ctx, self._stream, self.device)
            return _lib.MEM_DEVICE
        return _lib.MEM_HOST

    def _like(self, ref, n):
        if ref.dev:
            import torch
            return torch.empty(n, dtype=torch.float64, device=ref.obj.device)
        return np.empty(n)

    def profile(self, enable=True):
        """Start (or stop) per-kernel-family device timing with CUDA events."""
        self._check(self._lib.ins2d_profile(self._ctx, int(bool(enable))))

    def profile_read(self):
        """{family: (device ms, launches)} since the last read."""
        ms = (ctypes.c_double * len(_lib.PROF_FAMILIES))()
        n = (ctypes.c_int64 * len(_lib.PROF_FAMILIES))()
        self._check(self._lib.ins2d_profile_read(self._ctx, ms, n))
        return {f: (ms[i], int(n[i])) for i, f in enumerate(_lib.PROF_FAMILIES)}

    def set_stream(self, stream):
        """Issue work on a CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(self._lib.ins2d_set_stream(self._ctx, ctypes.c_void_p(stream)))
        self._stream = int(stream) if stream else None

    # -- boundary conditions ----------------------------------------------------
    def bc_samples(self, t):
        """The samples set_bc_vectors.m:52-79 takes from uBC/vBC at time t."""
        x, y, xp, yp, xin, yin = self.x, self.y, self.xp, self.yp, self.xin, self.yin
        u, v = self.uBC, self.vBC
        s = dict(uLo=u(x, y[0], t), uUp=u(x, y[-1], t), uLo_i=u(xin, y[0], t), uUp_i=u(xin, y[-1], t),
                 uLe_i=u(x[0], yp, t), uRi_i=u(x[-1], yp, t), vLe=v(x[0], y, t), vRi=v(x[-1], y, t),
                 vLo_i=v(xp, y[0], t), vUp_i=v(xp, y[-1], t), vLe_i=v(x[0], yin, t), vRi_i=v(x[-1], yin, t))
        pLe, pRi, pLo, pUp = self.pbc
        s.update(pLe=np.broadcast_to(pLe, (len(yp),)), pRi=np.broadcast_to(pRi, (len(yp),)),
                 pLo=np.broadcast_to(pLo, (len(xp),)), pUp=np.broadcast_to(pUp, (len(xp),)))
        if self.BC_unsteady:
            s.update(dudtLe_i=self.dudtBC(x[0], yp, t), dudtRi_i=self.dudtBC(x[-1], yp, t),
                     dvdtLo_i=self.dvdtBC(xp, y[0], t), dvdtUp_i=self.dvdtBC(xp, y[-1], t))
        return {k: np.ascontiguousarray(np.asarray(v_, dtype=np.float64).ravel()) for k, v_ in s.items()}

    def set_bc_vectors(self, t):
        """set_bc_vectors(t,options): samples the boundary functions and sends
        them to the device."""
        s = self.bc_samples(t)
        vals = _lib.BcValues()
        keep = []
        for name in _lib.BC_VALUE_FIELDS:
            if name in s:
                arr = s[name]
                keep.append(arr)
                setattr(vals, name, arr.ctypes.data_as(_lib.c_double_p))
        self._check(self._lib.ins2d_set_bc_values(self._ctx, float(t), ctypes.byref(vals)))

    # -- hot path ----------------------------------------------------------------
    def F(self, V, C=None, p=None, t=0.0, nopressure=0):
        """[maxres, F] = F(V,C,p,T,t,options,0,nopressure)."""
        Va = _Arr(V, self.NV, "V")
        Ca = _Arr(C, self.NV, "C") if C is not None and C is not V else None
        pa = None if nopressure else _Arr(p, self.Np, "p")
        out = self._like(Va, self.NV)
        Oa = _Arr(out, self.NV, "F")
        mem = self._mem(Va, Ca, pa, Oa)
        mr = ctypes.c_double()
        self._check(self._lib.ins2d_F(self._ctx, Va.ptr, Ca.ptr if Ca else None, pa.ptr if pa else None, float(t),
                                      int(bool(nopressure)), Oa.ptr, ctypes.byref(mr), mem))
        return mr.value, out

    def divergence(self, V):
        """M*V + yM and its max (check_conservation.m:37)."""
        Va = _Arr(V, self.NV, "V")
        out = self._like(Va, self.Np)
        Oa = _Arr(out, self.Np, "f")
        md = ctypes.c_double()
        self._check(self._lib.ins2d_divergence(self._ctx, Va.ptr, Oa.ptr, ctypes.byref(md), self._mem(Va, Oa)))
        return out, md.value

    def laplacian(self, p):
        """A*p with A = M*diag(Om_inv)*G."""
        pa = _Arr(p, self.Np, "p")
        out = self._like(pa, self.Np)
        Oa = _Arr(out, self.Np, "Ap")
        self._check(self._lib.ins2d_laplacian(self._ctx, pa.ptr, Oa.ptr, self._mem(pa, Oa)))
        return out

    def pressure_poisson(self, f, t=0.0, return_stats=False):
        """dp = pressure_poisson(f,t,options)."""
        fa = _Arr(f, self.Np, "f")
        out = self._like(fa, self.Np)
        Oa = _Arr(out, self.Np, "dp")
        st = _lib.SolveStats()
        self._check(self._lib.ins2d_pressure_poisson(self._ctx, fa.ptr, Oa.ptr, ctypes.byref(st), self._mem(fa, Oa)))
        if return_stats:
            return out, dict(iters=st.iters, norm1=st.norm1, norm2=st.norm2)
        return out

    def pressure_additional_solve(self, V, p, t=0.0, return_stats=False):
        """p = pressure_additional_solve(V,p,T,t,options) (returns a new p for
        host arrays, updates a device p in place)."""
        Va = _Arr(V, self.NV, "V")
        pa = _Arr(p if _is_torch_cuda(p) else np.array(p, dtype=np.float64), self.Np, "p")
        st = _lib.SolveStats()
        self._check(self._lib.ins2d_pressure_additional_solve(self._ctx, Va.ptr, pa.ptr, float(t), ctypes.byref(st),
                                                              self._mem(Va, pa)))
        if return_stats:
            return pa.obj, dict(iters=st.iters, norm1=st.norm1, norm2=st.norm2)
        return pa.obj

    def time_ERK(self, Vn, pn, tn, dt, nsteps=1, return_stats=False):
        """[Vnew, pnew] = time_ERK(Vn,pn,Tn,tn,dt,options); with nsteps > 1 the
        solver_unsteady.m time loop of that many steps.  Host arrays are
        copied (inputs untouched); device tensors are updated in place."""
        if _is_torch_cuda(Vn):
            Va, pa = _Arr(Vn, self.NV, "V"), _Arr(pn, self.Np, "p")
        else:
            Va = _Arr(np.array(Vn, dtype=np.float64), self.NV, "V")
            pa = _Arr(np.array(pn, dtype=np.float64), self.Np, "p")
        st = _lib.StepStats()
        self._check(self._lib.ins2d_erk_run(self._ctx, Va.ptr, pa.ptr, float(tn), float(dt), int(nsteps),
                                            ctypes.byref(st), self._mem(Va, pa)))
        if return_stats:
            return Va.obj, pa.obj, dict(n_solves=st.n_solves, iters_total=st.iters_total, iters_max=st.iters_max,
                                        norm1_max=st.norm1_max)
        return Va.obj, pa.obj

    def check_conservation(self, V, t=0.0):
        """[maxdiv, umom, vmom, k] = check_conservation(V,T,t,options)."""
        Va = _Arr(V, self.NV, "V")
        out = (ctypes.c_double * 4)()
        self._check(self._lib.ins2d_conservation(self._ctx, Va.ptr, float(t), out, self._mem(Va)))
        return tuple(out)

    def initial_projection(self, V, t=0.0, return_maxdiv=False):
        """input_check.m:95-111: project V when max|M V + yM| > 1e-12 (a new
        array for host input, a device tensor in place)."""
        Va = _Arr(V if _is_torch_cuda(V) else np.array(V, dtype=np.float64), self.NV, "V")
        md = ctypes.c_double()
        self._check(self._lib.ins2d_initial_projection(self._ctx, Va.ptr, float(t), ctypes.byref(md),
                                                       self._mem(Va)))
        if return_maxdiv:
            return Va.obj, md.value
        return Va.obj


class Ensemble:
    """Independent flows advanced together (ins2d_ens_*): ``members`` is a
    list of dicts of :class:`Options` keyword arguments (x, y, BC, Re, uBC,
    vBC, CG_acc, ...); every phase of a time step is one launch over all
    members and the Poisson solves one persistent launch.  ``member(m)`` is
    the member's :class:`Options` (its F, conservation, boundary values);
    the ensemble holds each member's state (set_state / get_state)."""

    def __init__(self, members):
        self._lib = _lib.load()
        self.members = []
        self._stream = None
        self._device = int(members[0].get("device", 0)) if members else 0
        # describe every member with an Options-like set of descriptors (no
        # context is created for the descriptors themselves)
        descs = [_describe(**kw) for kw in members]
        n = len(descs)
        G = (_lib.GridDesc * n)(*[d[0] for d in descs])
        B = (_lib.BcDesc * n)(*[d[1] for d in descs])
        O = (_lib.Opts * n)(*[d[2] for d in descs])
        self._keep = descs
        self._e = ctypes.c_void_p()
        rc = self._lib.ins2d_ens_create(n, G, B, O, ctypes.byref(self._e))
        if rc != 0:
            msg = self._lib.ins2d_ens_last_error(self._e)
            self._lib.ins2d_ens_destroy(self._e)
            self._e = None
            raise Ins2dError(rc, msg.decode() if msg else "")
        for m, kw in enumerate(members):
            h = self._lib.ins2d_ens_member(self._e, m)
            opts = Options(_handle=h, **kw)
            opts.set_bc_vectors(0.0)
            self.members.append(opts)

    def __len__(self):
        return len(self.members)

    def member(self, m):
        return self.members[m]

    def _check(self, rc):
        if rc != 0:
            msg = self._lib.ins2d_ens_last_error(self._e)
            raise Ins2dError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_e", None):
            for o in self.members:
                o._ctx = None
            self._lib.ins2d_ens_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        self._check(self._lib.ins2d_ens_set_stream(self._e, ctypes.c_void_p(stream)))
        self._stream = int(stream) if stream else None

    def _mem(self, *arrs):
        kinds = {a.dev for a in arrs if a is not None}
        if len(kinds) > 1:
            raise ValueError("mix of host and device arrays")
        if kinds == {True}:
            _order_after_torch(self._lib.ins2d_ens_wait_stream, self._e, self._stream, self._device)
            return _lib.MEM_DEVICE
        return _lib.MEM_HOST

    def set_state(self, m, V, p):
        o = self.members[m]
        Va, pa = _Arr(V, o.NV, "V"), _Arr(p, o.Np, "p")
        self._check(self._lib.ins2d_ens_set_state(self._e, m, Va.ptr, pa.ptr, self._mem(Va, pa)))

    def set_member_dt(self, m, dt):
        """Give member m its own time step (0: the run's dt)."""
        self._check(self._lib.ins2d_ens_set_member_dt(self._e, m, float(dt)))

    def get_state(self, m, V=None, p=None):
        """The member's (V, p), into the given host arrays when passed."""
        o = self.members[m]
        V = np.empty(o.NV) if V is None else V
        p = np.empty(o.Np) if p is None else p
        Va, pa = _Arr(V, o.NV, "V"), _Arr(p, o.Np, "p")
        for a, arr in ((Va, V), (pa, p)):
            if not a.dev and (not isinstance(arr, np.ndarray) or a.ptr != arr.ctypes.data):
                raise ValueError("get_state: output arrays must be contiguous float64")
        self._check(self._lib.ins2d_ens_get_state(self._e, m, Va.ptr, pa.ptr, self._mem(Va, pa)))
        return V, p

    def state_tensors(self, m):
        """The member's device state as (V, p) torch CUDA tensors (views)."""
        import torch
        Vp, pp = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self._lib.ins2d_ens_state_ptr(self._e, m, ctypes.byref(Vp), ctypes.byref(pp)))
        o = self.members[m]
        return _cuda_view(Vp.value, o.NV), _cuda_view(pp.value, o.Np)

    def time_ERK(self, t, dt, nsteps=1):
        """nsteps of time_ERK for every member; returns per-member stats."""
        n = len(self.members)
        st = (_lib.StepStats * n)()
        self._check(self._lib.ins2d_ens_erk_run(self._e, float(t), float(dt), int(nsteps), st))
        return [dict(n_solves=s.n_solves, iters_total=s.iters_total, iters_max=s.iters_max, norm1_max=s.norm1_max)
                for s in st]

    def set_solver(self, threads):
        """-1: tuned on the first run; 0: batched across members; 256/512:
        persistent launch with that many threads per member."""
        self._check(self._lib.ins2d_ens_set_solver(self._e, int(threads)))

    def solve_shape(self):
        th, bl = ctypes.c_int32(), ctypes.c_int32()
        ms = (ctypes.c_double * 3)()
        self._check(self._lib.ins2d_ens_solve_shape(self._e, ctypes.byref(th), ctypes.byref(bl), ms))
        return dict(threads=th.value, blocks=bl.value, batched=th.value == 0,
                    tuned_ms={"persistent512": ms[0], "persistent256": ms[1], "batched": ms[2]})


def _describe(x, y, BC, Re=1000.0, poisson=4, CG_acc=1e-12, CG_maxit=10000, p_add_solve=1, RK="RK44",
              precision="fp64", device=0, precond="default", **_ignored):
    """C descriptors (grid, BC, options) of one case, as Options builds them."""
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    y = np.ascontiguousarray(np.asarray(y, dtype=np.float64))
    g = _lib.GridDesc(len(x) - 1, len(y) - 1, x.ctypes.data_as(_lib.c_double_p), y.ctypes.data_as(_lib.c_double_p))
    codes = [_lib.BC_CODES[BC[c][sd]] for c in ("u", "v") for sd in ("left", "right", "low", "up")]
    b = _lib.BcDesc(*codes, int(BC.get("BC_unsteady", 0)))
    o = _lib.Opts()
    o.Re = float(Re)
    o.poisson = int(poisson)
    o.CG_acc = float(CG_acc)
    o.CG_maxit = int(CG_maxit)
    o.p_add_solve = int(p_add_solve)
    A, bb, c = getRKmethod(RK)
    s = len(bb)
    o.rk_stages = s
    for i in range(s):
        for j in range(s):
            o.rk_A[i * s + j] = A[i, j]
        o.rk_b[i] = bb[i]
        o.rk_c[i] = c[i]
    o.precision = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32_STENCIL}[precision]
    o.device = int(device)
    o.precond = _lib.PRECOND_CODES[precond]
    return g, b, o, x, y


def _order_after_torch(wait_fn, handle, stream, device):
    """Makes the library's stream wait for the work queued so far on torch's
    current stream of `device` (a no-op when the library was given that very
    stream through set_stream)."""
    import torch
    cur = torch.cuda.current_stream(device).cuda_stream
    if stream is not None and int(stream) == int(cur):
        return
    rc = wait_fn(handle, ctypes.c_void_p(cur))
    if rc != 0:
        raise Ins2dError(rc, "ordering the library's stream after torch's current stream failed")


def _cuda_view(ptr, n):
    """A float64 CUDA tensor viewing n values at a device pointer."""
    import torch

    class _Iface:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2}

    return torch.as_tensor(_Iface(), device="cuda")


# -- module-level functions with the reference's names ------------------------------
def F(V, C, p, T, t, options, getJacobian=0, nopressure=0):
    """[maxres,F,dF] = F(V,C,p,T,t,options,getJacobian,nopressure); the
    Jacobian is not part of this path (dF is None)."""
    if getJacobian:
        raise NotImplementedError("the Jacobian of F is not part of the explicit path")
    maxres, Fv = options.F(V, C, p, t, nopressure)
    return maxres, Fv, None


def pressure_poisson(f, t, options):
    return options.pressure_poisson(f, t)


def pressure_additional_solve(V, p, T, t, options):
    return options.pressure_additional_solve(V, p, t)


def time_ERK(Vn, pn, Tn, tn, dt, options):
    V, p = options.time_ERK(Vn, pn, tn, dt)
    return V, p, 0


def check_conservation(V, T, t, options):
    return options.check_conservation(V, t)
