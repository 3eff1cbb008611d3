"""ffcm_b200 -- B200 (sm_100a) backend of the FFCM mobility operator.

A host-side mirror of the reference Julia API of ForceCouplingMethod.jl
(Biofluid-Dynamics-Group/FFCM.jl) over the C ABI of libffcm_b200.so:

=========================================  =========================================
reference (Julia)                          here (Python)
=========================================  =========================================
``FFCMConfig{T}(; L, R_c, N, ...)``        ``FFCMConfig(T, L=..., R_c=..., N=..., ...)``
``mobility!(V, config, Y, F)``             ``mobility(V, config, Y, F)``
``FFCMMobility(config, Y)``                ``FFCMMobility(config, Y)``
``mul!(v, M, f)`` / ``mul!(v, M, f, a, b)``  ``M.mul(v, f)`` / ``M.mul(v, f, a, b)``
``M * F``                                  ``M @ F`` (also ``M * F``)
``wrap_positions!`` ... ``correct_velocities!``  same names without ``!``
=========================================  =========================================

Array convention: a Julia ``3xN`` column-major matrix is a NumPy ``(N, 3)``
C-order array (the same bytes); shapes are checked in Julia's ``(rows, cols)``
terms, so an ``(N, 3)`` array is ``3xN``. Arrays may be NumPy arrays (host
memory; the call copies through the device and returns when V is ready) or
CUDA ``torch.Tensor`` s of the same shape (device memory; the call is
asynchronous on the current torch stream). Index buffers are 1-based, as in
Julia. Errors mirror the reference: ``ArgumentError`` for invalid parameters
(src/config.jl:267-312), ``DimensionMismatch`` for shapes
(src/mobility.jl:29-34).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L_

__all__ = ["FFCMConfig", "mobility", "FFCMMobility", "FFCMBatch", "ArgumentError", "DimensionMismatch",
           "FFCMError", "wrap_positions", "assign_cells", "sort_particles_by_cell",
           "spread_forces", "stokes_solve", "interpolate_velocities", "correct_velocities",
           "mobility_checkpoint", "adjoint", "objective_gradient", "rrule_mobility",
           "mobility_autograd", "cg", "CGHistory", "wisdom_export", "wisdom_import", "batch_offsets",
           "pack_batch", "unpack_batch", "dist_partition", "DistributedConfig", "TorchExchange", "LocalExchange",
           "distributed_mobility_local"]


class ArgumentError(ValueError):
    """Invalid configuration parameter (Julia ArgumentError)."""


class DimensionMismatch(ValueError):
    """Array shape does not match the configuration (Julia DimensionMismatch)."""


class FFCMError(RuntimeError):
    """CUDA, allocation, timeout or state error reported by the library."""


def _raise(code: int):
    if code == L_.OK:
        return
    msg = L_.last_error()
    if code == L_.ERR_ARGUMENT:
        raise ArgumentError(msg)
    if code == L_.ERR_DIMENSION:
        raise DimensionMismatch(msg)
    if code == L_.ERR_OOM:
        raise MemoryError(msg)
    raise FFCMError(f"[status {code}] {msg}")


def _dtype_code(T):
    T = np.dtype(T)
    if T == np.float32:
        return L_.FLOAT32
    if T == np.float64:
        return L_.FLOAT64
    raise ArgumentError(f"working precision must be Float32 or Float64; got {T}")


def _dptr(vals):
    arr = (ctypes.c_double * len(vals))(*[float(v) for v in vals])
    return arr


def _i32ptr(vals):
    return (ctypes.c_int32 * len(vals))(*[int(v) for v in vals])


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _julia_size(x):
    """Julia (rows, cols) of an (N, 3)-style row-major array."""
    shape = tuple(x.shape)
    if len(shape) == 2:
        return shape[1], shape[0]
    if len(shape) == 1:
        return shape[0], 1
    return (-1, -1)


class _Arg:
    """A particle array handed to the C ABI (pointer, memory kind, keep-alive)."""

    def __init__(self, x, T, writable=False, device=None):
        self.src = x
        if _is_torch(x):
            import torch
            if x.dtype != (torch.float32 if T == np.float32 else torch.float64):
                raise ArgumentError(f"tensor dtype {x.dtype} does not match the config's {np.dtype(T)}")
            if not x.is_contiguous():
                raise ArgumentError("tensors must be contiguous")
            if x.is_cuda and device is not None and x.device.index != int(device):
                # the library's kernels run on the configuration's GPU; another
                # GPU's memory would fault there instead of raising
                raise ArgumentError(f"tensor lives on cuda:{x.device.index}, the configuration on "
                                    f"cuda:{int(device)}")
            self.memory = L_.DEVICE if x.is_cuda else L_.HOST
            self.ptr = x.data_ptr()
            self.buf = x
            self.copy_back = None
        else:
            a = np.asarray(x)
            if a.dtype != np.dtype(T):
                raise ArgumentError(f"array dtype {a.dtype} does not match the config's {np.dtype(T)}")
            if writable:
                if not a.flags.c_contiguous or not a.flags.writeable:
                    raise ArgumentError("V must be a writable C-contiguous array")
                buf = a
            else:
                buf = np.ascontiguousarray(a)
            self.memory = L_.HOST
            self.ptr = buf.ctypes.data
            self.buf = buf
        self.rows, self.cols = _julia_size(x)


# cudaStreamLegacy: the legacy default stream. torch reports its default stream
# as handle 0, which the C ABI reads as "the configuration's own stream".
_CUDA_STREAM_LEGACY = 1


def _stream_handle(s):
    """A cudaStream_t for the C ABI from a torch stream or a raw handle."""
    h = int(getattr(s, "cuda_stream", s) or 0)
    return ctypes.c_void_p(h if h != 0 else _CUDA_STREAM_LEGACY)


def _stream_of(*args):
    for a in args:
        if a is not None and a.memory == L_.DEVICE:
            import torch
            return _stream_handle(torch.cuda.current_stream(a.src.device))
    return None


class FFCMConfig:
    """B200 counterpart of ``FFCMConfig{T}`` (src/config.jl:466-546).

    Validates the parameters exactly as the reference (same order, same
    ArgumentError conditions), derives the scalars in precision ``T`` and
    allocates every hot-path buffer on ``device``. ``N`` is fixed at
    construction. ``fft_planning`` and ``fft_threads`` are validated and then
    have no effect (they configure FFTW on the reference's CPU backend).
    ``gpu_acceleration`` must be true: this configuration always lives on the
    GPU; the CPU backend is the reference's own.

    ``stencil`` (no reference counterpart): ``"reference"`` (default) picks
    each stencil's anchor and offsets with the reference's arithmetic in
    precision T, so results match its CPU backend to round-off; ``"float64"``
    picks them in double precision from the box length as given
    (``ffcm_set_stencil``), which keeps Float32 results at the Float64 answer
    where Float32 anchors would flip (large boxes). ``None`` keeps the
    library's default (the ``FFCM_STENCIL`` environment variable, else
    ``"reference"``).
    """

    def __init__(self, T=np.float32, *, L, R_c, N, a=1.0, kernel_widths_ratio,
                 num_grid_points, M_G, viscosity, fft_planning="measure", fft_threads=1,
                 gpu_acceleration=True, device=0, stencil=None):
        self._h = None
        self.T = np.dtype(T).type
        dt = _dtype_code(T)
        if not gpu_acceleration:
            raise ArgumentError("this backend builds configurations on the GPU only; "
                                "use the reference CPU backend for gpu_acceleration = false")
        if fft_planning not in L_.FFT_PLANNING:
            raise ArgumentError(f"fft_planning must be :estimate, :measure, or :patient; got "
                                f":{fft_planning}")
        lib = L_.load()
        Lp = _dptr(L)
        Mp = _i32ptr(num_grid_points)
        h = ctypes.c_void_p()
        _raise(lib.ffcm_create(ctypes.byref(h), dt, Lp, float(R_c), int(N), float(a),
                               float(kernel_widths_ratio), Mp, int(M_G), float(viscosity),
                               L_.FFT_PLANNING[fft_planning], int(fft_threads), int(device)))
        self._h = h
        self.device = int(device)
        self.N = int(N)
        T_ = self.T
        self.L = tuple(T_(x) for x in L)
        self.R_c = T_(R_c)
        self.a = T_(a)
        self.mu = T_(viscosity)
        self.num_grid_points = tuple(int(m) for m in num_grid_points)
        self.M_G = int(M_G)
        nc = (ctypes.c_int32 * 3)()
        cs = (ctypes.c_double * 3)()
        ics = (ctypes.c_double * 3)()
        s, S, hh, ih = (ctypes.c_double() for _ in range(4))
        _raise(lib.ffcm_derive_scalars(dt, Lp, float(R_c), float(a), float(kernel_widths_ratio),
                                       Mp, nc, cs, ics, ctypes.byref(s), ctypes.byref(S),
                                       ctypes.byref(hh), ctypes.byref(ih)))
        self.num_cells = tuple(int(v) for v in nc)
        self.cell_size = tuple(T_(v) for v in cs)
        self.inv_cell_size = tuple(T_(v) for v in ics)
        self.sigma, self.Sigma = T_(s.value), T_(S.value)
        self.h, self.inv_h = T_(hh.value), T_(ih.value)
        self.num_cells_total = int(np.prod(self.num_cells))
        if stencil is not None:
            self.stencil = stencil

    @property
    def stencil(self):
        """``"reference"`` or ``"float64"`` (see the class docstring)."""
        m = ctypes.c_int32(0)
        _raise(L_.load().ffcm_get_stencil(self.handle, ctypes.byref(m)))
        return {v: k for k, v in L_.STENCIL.items()}[m.value]

    @stencil.setter
    def stencil(self, mode):
        if mode not in L_.STENCIL:
            raise ArgumentError(f"stencil must be 'reference' or 'float64'; got {mode!r}")
        _raise(L_.load().ffcm_set_stencil(self.handle, L_.STENCIL[mode]))

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            L_.load().ffcm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if not self._h:
            raise FFCMError("configuration has been closed")
        return self._h

    # -- buffers in the reference layouts --------------------------------
    def _buf_shape(self, name):
        N, M, nc = self.N, self.num_grid_points, self.num_cells_total
        T = self.T
        return {
            "Y_WRAPPED": ((N, 3), T), "Y_SORTED": ((N, 3), T), "F_SORTED": ((N, 3), T),
            "CELL_HASH": ((N,), np.int32), "ORIGINAL_INDEX": ((N,), np.int32),
            "CELL_START": ((nc,), np.int32), "CELL_END": ((nc,), np.int32),
            "FORCE_DENSITY": ((3, M[2], M[1], M[0]), T),
            "FLUID_VELOCITY": ((3, M[2], M[1], M[0]), T),
            "K_X": ((M[0] // 2 + 1,), T), "K_Y": ((M[1],), T), "K_Z": ((M[2],), T),
            "NEIGHBOR_MAP": ((13 * nc,), np.int32),
        }[name]

    def get(self, name):
        """Copy a configuration buffer to a new NumPy array (reference layout)."""
        name = name.upper()
        shape, dt = self._buf_shape(name)
        out = np.empty(shape, dt)
        _raise(L_.load().ffcm_get_buffer(self.handle, L_.BUF[name], out.ctypes.data, out.nbytes,
                                         L_.HOST, None))
        return out

    def set(self, name, value):
        """Overwrite a configuration buffer from a NumPy array (reference layout)."""
        name = name.upper()
        shape, dt = self._buf_shape(name)
        arr = np.ascontiguousarray(np.asarray(value, dt).reshape(shape))
        _raise(L_.load().ffcm_set_buffer(self.handle, L_.BUF[name], arr.ctypes.data, arr.nbytes,
                                         L_.HOST, None))

    # reference-style accessors
    cell_hash = property(lambda self: self.get("CELL_HASH"))
    original_index = property(lambda self: self.get("ORIGINAL_INDEX"))
    cell_start = property(lambda self: self.get("CELL_START"))
    cell_end = property(lambda self: self.get("CELL_END"))
    Y_wrapped = property(lambda self: self.get("Y_WRAPPED"))
    Y_sorted = property(lambda self: self.get("Y_SORTED"))
    F_sorted = property(lambda self: self.get("F_SORTED"))
    force_density = property(lambda self: self.get("FORCE_DENSITY"))
    fluid_velocity = property(lambda self: self.get("FLUID_VELOCITY"))
    k_x = property(lambda self: self.get("K_X"))
    k_y = property(lambda self: self.get("K_Y"))
    k_z = property(lambda self: self.get("K_Z"))

    # -- measurement --------------------------------------------------------
    def profile_begin(self):
        _raise(L_.load().ffcm_profile_begin(self.handle))

    def profile_end(self):
        ms = (ctypes.c_double * len(L_.STAGES))()
        calls = (ctypes.c_int64 * len(L_.STAGES))()
        _raise(L_.load().ffcm_profile_end(self.handle, ms, calls))
        return {name: (ms[i], calls[i]) for i, name in enumerate(L_.STAGES)}

    def tuning(self):
        """The y/z pass variant this configuration uses (the autotuner's, or
        a reused / imported choice): a dict of `ffcm_get_tuning`'s fields."""
        out = (ctypes.c_int32 * 7)()
        _raise(L_.load().ffcm_get_tuning(self.handle, out))
        names = ("y_kind", "y_columns", "y_grid", "z_kind", "z_columns", "z_grid", "kx_chunk")
        return dict(zip(names, (int(x) for x in out)))

    def launch_count(self):
        return int(L_.load().ffcm_launch_count(self.handle))

    def synchronize(self):
        _raise(L_.load().ffcm_synchronize(self.handle, None))


def mobility(V, config: FFCMConfig, Y, F, stream=None):
    """``mobility!(V, config, Y, F) -> V`` (src/mobility.jl:23-45).

    Overwrites V with the velocities induced by forces F at positions Y, in
    the caller's original particle order. Y and F are never modified.
    ``stream`` (a cudaStream_t as int, or a torch.cuda.Stream) overrides the
    stream the call runs on: by default the current torch stream for CUDA
    tensors and the configuration's own stream for host arrays.
    """
    T = config.T
    for x in (V, Y, F):
        if len(getattr(x, "shape", ())) != 2:
            raise DimensionMismatch(
                f"V, Y, and F must each be 3xN for the config's N = {config.N}")
    v = _Arg(V, T, writable=True, device=config.device)
    y = _Arg(Y, T, device=config.device)
    f = _Arg(F, T, device=config.device)
    if len({v.memory, y.memory, f.memory}) != 1:
        raise ArgumentError("V, Y and F must all be host arrays or all be CUDA tensors")
    if stream is None:
        st = _stream_of(v)
    else:
        st = _stream_handle(stream)
    _raise(L_.load().ffcm_mobility(config.handle, v.ptr, v.rows, v.cols, y.ptr, y.rows, y.cols,
                                   f.ptr, f.rows, f.cols, v.memory, st))
    return V


# ---- the six steps (reference src/cell_list.jl ... src/correct_velocities.jl) ----

def wrap_positions(config: FFCMConfig, Y):
    """``wrap_positions!(config.particles.Y_wrapped, Y, config.L)``."""
    y = _Arg(Y, config.T, device=config.device)
    if (y.rows, y.cols) != (3, config.N):
        raise DimensionMismatch("Y must be 3xN")
    _raise(L_.load().ffcm_wrap_positions(config.handle, y.ptr, y.memory, _stream_of(y)))
    return config


def assign_cells(config: FFCMConfig):
    """``assign_cells!(config, config.particles.Y_wrapped)``."""
    _raise(L_.load().ffcm_assign_cells(config.handle, None))
    return config


def sort_particles_by_cell(config: FFCMConfig, F):
    """``sort_particles_by_cell!(config, config.particles.Y_wrapped, F)``."""
    f = _Arg(F, config.T, device=config.device)
    if (f.rows, f.cols) != (3, config.N):
        raise DimensionMismatch("F must be 3xN")
    _raise(L_.load().ffcm_sort_particles_by_cell(config.handle, f.ptr, f.memory, _stream_of(f)))
    return config


def spread_forces(config: FFCMConfig):
    """``spread_forces!(config)``."""
    _raise(L_.load().ffcm_spread_forces(config.handle, None))
    return config


def stokes_solve(config: FFCMConfig):
    """``stokes_solve!(config)``."""
    _raise(L_.load().ffcm_stokes_solve(config.handle, None))
    return config


def interpolate_velocities(V, config: FFCMConfig):
    """``interpolate_velocities!(V, config)`` (overwrites V, original order)."""
    v = _Arg(V, config.T, writable=True, device=config.device)
    if (v.rows, v.cols) != (3, config.N):
        raise DimensionMismatch("V must be 3xN")
    _raise(L_.load().ffcm_interpolate_velocities(config.handle, v.ptr, v.memory, _stream_of(v)))
    return V


def correct_velocities(V, config: FFCMConfig):
    """``correct_velocities!(V, config)`` (adds to V)."""
    v = _Arg(V, config.T, writable=True, device=config.device)
    if (v.rows, v.cols) != (3, config.N):
        raise DimensionMismatch("V must be 3xN")
    _raise(L_.load().ffcm_correct_velocities(config.handle, v.ptr, v.memory, _stream_of(v)))
    return V


def _torch_empty_particles(F, config):
    """An (N, 3) CUDA tensor of the config's type on F's device."""
    import torch
    dt = torch.float32 if np.dtype(config.T) == np.float32 else torch.float64
    return torch.empty((config.N, 3), dtype=dt, device=F.device)


class FFCMMobility:
    """Matrix-free operator ``FFCMMobility(config, Y)`` (src/mobility.jl:88-155).

    ``size`` is ``(3N, 3N)`` on the flat column-major view (entry 3(n-1)+i is
    axis i of particle n). ``mul(v, f)`` applies it, ``mul(v, f, alpha, beta)``
    computes ``alpha*M*f + beta*v`` (beta = 0 overwrites v, ignoring NaN
    contents), ``M @ F`` maps a 3xN force array to a fresh velocity array.
    Symmetric positive-definite by construction.

    The positions are fixed once: their cell list is built at construction
    (``ffcm_set_positions``) and every application only re-gathers the forces
    (``ffcm_mobility_apply``). If another solve ran on ``config`` in between,
    the positions are fixed again before the application. Y, and the forces
    of ``M @ F`` / ``mul``, may be CUDA tensors: they are then used in place on
    the current torch stream (no host staging).
    """

    def __init__(self, config: FFCMConfig, Y):
        if not _is_torch(Y):
            Y = np.asarray(Y)
        r, c = _julia_size(Y)
        if r != 3:
            raise ArgumentError(f"Y must be 3xN; got size ({r}, {c})")
        if c != config.N:
            raise ArgumentError(f"Y has {c} particles but config was built for {config.N}; "
                                "construct a config with matching N")
        self.config = config
        if _is_torch(Y):
            # a CUDA tensor stays on the device (a private copy: Y is never mutated)
            self.Y = _Arg(Y, config.T, device=config.device).buf.detach().clone()
        else:
            self.Y = np.ascontiguousarray(Y, config.T).copy()
        self.F_scratch = np.empty((config.N, 3), config.T)
        self.V_scratch = np.empty((config.N, 3), config.T)
        self._set_positions()

    def _set_positions(self):
        y = _Arg(self.Y, self.config.T, device=self.config.device)
        _raise(L_.load().ffcm_set_positions(self.config.handle, y.ptr, y.memory, _stream_of(y)))

    def _apply(self, V, F):
        """V = M F for (N, 3) host arrays of the config's type."""
        lib = L_.load()
        code = lib.ffcm_mobility_apply(self.config.handle, V.ctypes.data, F.ctypes.data, L_.HOST, None)
        if code == L_.ERR_STATE:     # the config solved something else since
            self._set_positions()
            code = lib.ffcm_mobility_apply(self.config.handle, V.ctypes.data, F.ctypes.data, L_.HOST, None)
        _raise(code)
        return V

    @property
    def shape(self):
        n = 3 * self.config.N
        return (n, n)

    def size(self, d=None):
        n = 3 * self.config.N
        if d is None:
            return (n, n)
        return n if d <= 2 else 1

    @property
    def dtype(self):
        return np.dtype(self.config.T)

    def _apply_device(self, V, F):
        """V = M F for (N, 3) CUDA tensors of the config's type: zero copy, on
        the current torch stream (the device fast path the reference's
        `mul!` lacks: it stages through host arrays, src/mobility.jl:115-147)."""
        v, f = _particle_args(self.config, (("V", V), ("F", F)), writable=("V",))
        st = _stream_of(v)
        lib = L_.load()
        code = lib.ffcm_mobility_apply(self.config.handle, v.ptr, f.ptr, v.memory, st)
        if code == L_.ERR_STATE:     # the config solved something else since
            self._set_positions()
            code = lib.ffcm_mobility_apply(self.config.handle, v.ptr, f.ptr, v.memory, st)
        _raise(code)
        return V

    def mul(self, v, f, alpha=None, beta=None):
        T = self.config.T
        if _is_torch(f) and f.is_cuda:
            # the operator's element type, as the reference's mul! converts
            # (copyto! into its T scratch, src/mobility.jl:115-147)
            ft = f.to(_torch_empty_particles(f, self.config).dtype)
            out = _torch_empty_particles(f, self.config)
            self._apply_device(out, ft.reshape(self.config.N, 3).contiguous())
            out = out.reshape(-1)
            if not _is_torch(v):
                # a host v: bring the result over and finish on the host
                res = out.cpu().numpy()
                vv = np.asarray(v)
                if alpha is None and beta is None:
                    np.copyto(vv, res.reshape(vv.shape), casting="same_kind")
                    return v
                a = T(1 if alpha is None else alpha)
                b = T(0 if beta is None else beta)
                np.copyto(vv, (a * res if b == 0 else a * res + b * vv.reshape(-1)).reshape(vv.shape),
                          casting="same_kind")
                return v
            if alpha is None and beta is None:
                v.copy_(out.reshape(v.shape))
                return v
            a = 1.0 if alpha is None else float(alpha)
            b = 0.0 if beta is None else float(beta)
            res = a * out if b == 0 else a * out + b * v.reshape(-1)
            v.copy_(res.reshape(v.shape))
            return v
        self.F_scratch[...] = np.asarray(f, T).reshape(self.config.N, 3)
        self._apply(self.V_scratch, self.F_scratch)
        out = self.V_scratch.reshape(-1)
        if alpha is None and beta is None:
            v[...] = out
            return v
        a = T(1 if alpha is None else alpha)
        b = T(0 if beta is None else beta)
        if b == 0:
            v[...] = a * out
        else:
            v[...] = a * out + b * v
        return v

    def __matmul__(self, F):
        if _is_torch(F) and F.is_cuda:
            if len(F.shape) != 2 or _julia_size(F) != (3, self.config.N):
                raise DimensionMismatch(f"F must be 3xN for the config's N = {self.config.N}")
            return self._apply_device(_torch_empty_particles(F, self.config), F.contiguous())
        F = np.asarray(F)
        if len(F.shape) != 2 or _julia_size(F) != (3, self.config.N):
            raise DimensionMismatch(f"F must be 3xN for the config's N = {self.config.N}")
        V = np.empty((self.config.N, 3), self.config.T)
        return self._apply(V, np.ascontiguousarray(F, self.config.T))

    __mul__ = __matmul__

    @staticmethod
    def issymmetric():
        return True

    @staticmethod
    def isposdef():
        return True


# ---- launch-shape wisdom (the analogue of FFTW's exported wisdom) ----

def wisdom_export() -> str:
    """The autotuner's choices of this process as text (`ffcm_wisdom_export`)."""
    lib = L_.load()
    n = int(lib.ffcm_wisdom_export(None, 0))
    buf = ctypes.create_string_buffer(n + 1)
    lib.ffcm_wisdom_export(buf, n + 1)
    return buf.value.decode()


def wisdom_import(text: str):
    """Add choices from `wisdom_export` text; later configurations of those
    shapes on this machine skip the autotuner (`ffcm_wisdom_import`)."""
    _raise(L_.load().ffcm_wisdom_import(text.encode()))


# ---- resistance problem: conjugate gradients on the operator ----

class CGHistory:
    """What ``cg(...; log=true)`` of IterativeSolvers.jl reports and a caller
    reads: ``isconverged``, ``iters`` (iterations, one operator application
    each), ``resnorm`` (|r| of the recursion at the end) and ``status``
    ('converged', 'maxiter' or 'breakdown')."""

    def __init__(self, iters, resnorm, status):
        self.iters = int(iters)
        self.resnorm = float(resnorm)
        self.status = L_.CG_STATUS.get(int(status), f"status {int(status)}")
        self.isconverged = self.status == "converged"

    def __repr__(self):
        return f"CGHistory(iters={self.iters}, resnorm={self.resnorm:.3e}, status={self.status!r})"


def cg(M: FFCMMobility, V, *, reltol=None, abstol=0.0, maxiter=None, log=False, x0=None, out=None,
       stream=None):
    """Solve the resistance problem M(Y) F = V for F by conjugate gradients,
    the use the reference declares ``FFCMMobility`` symmetric positive definite
    for (src/mobility.jl:161-162; ``cg(M, V)`` of IterativeSolvers.jl in
    Julia). The whole iteration runs on the device (``ffcm_cg_solve``).

    Keywords as IterativeSolvers.jl's ``cg``: stop once
    |r| <= max(reltol |r0|, abstol) or after ``maxiter`` iterations;
    ``reltol`` defaults to sqrt(eps(T)), ``maxiter`` to 3N. ``x0`` is an
    initial guess (default zero, ``initially_zero``). ``V`` (and ``out``,
    ``x0``) are 3xN host arrays or all CUDA tensors of the config's type.
    Returns F, or ``(F, CGHistory)`` with ``log=True``.
    """
    config = M.config
    T = config.T
    if out is None:
        if _is_torch(V):
            import torch
            out = torch.empty_like(V)
        else:
            out = np.empty((config.N, 3), T)
    flags = 0
    if x0 is not None:
        out[...] = x0 if _is_torch(out) else np.asarray(x0, T).reshape(config.N, 3)
        flags = L_.CG_INITIAL_GUESS
    f, v = _particle_args(config, (("F", out), ("V", V)), writable=("F",))
    st = _stream_of(f) if stream is None else _stream_handle(stream)
    it, res, status = ctypes.c_int32(0), ctypes.c_double(0.0), ctypes.c_int32(0)
    rt = -1.0 if reltol is None else float(reltol)
    mi = -1 if maxiter is None else int(maxiter)
    lib = L_.load()

    def call():
        return lib.ffcm_cg_solve(config.handle, f.ptr, v.ptr, f.memory, rt, float(abstol), mi, flags,
                                 ctypes.byref(it), ctypes.byref(res), ctypes.byref(status), st)

    code = call()
    if code == L_.ERR_STATE:     # the config solved something else since
        M._set_positions()
        code = call()
    _raise(code)
    if log:
        return out, CGHistory(it.value, res.value, status.value)
    return out


# ---- adjoint form (no reference counterpart: the reference has no derivative) ----

def _particle_args(config, named, writable=()):
    """_Arg per (name, array); all 3xN of the config's N, one memory kind."""
    T = config.T
    args = []
    for name, x in named:
        if len(getattr(x, "shape", ())) != 2:
            raise DimensionMismatch(f"{name} must be 3xN for the config's N = {config.N}")
        a = _Arg(x, T, writable=name in writable, device=config.device)
        if (a.rows, a.cols) != (3, config.N):
            raise DimensionMismatch(f"{name} must be 3xN for the config's N = {config.N}; "
                                    f"got size ({a.rows}, {a.cols})")
        args.append(a)
    if len({a.memory for a in args}) != 1:
        raise ArgumentError("all arrays must be host arrays or all be CUDA tensors")
    return args


def mobility_checkpoint(V, config: FFCMConfig, Y, F, stream=None):
    """``mobility!`` that also keeps what the pullback needs (the velocity grid
    u = L^-1 S F, the cell list and the sorted particles) on the config."""
    v, y, f = _particle_args(config, (("V", V), ("Y", Y), ("F", F)), writable=("V",))
    st = _stream_of(v) if stream is None else _stream_handle(stream)
    _raise(L_.load().ffcm_mobility_checkpoint(config.handle, v.ptr, y.ptr, f.ptr, v.memory, st))
    return V


def adjoint(dY, dF, config: FFCMConfig, lam, stream=None):
    """Pullback of the last ``mobility_checkpoint`` on ``config`` at the
    cotangent ``lam`` = dJ/dV: writes dJ/dY into ``dY`` and dJ/dF = M lam into
    ``dF`` (3xN each). Raises FFCMError if another solve ran since."""
    gy, gf, l_ = _particle_args(config, (("dY", dY), ("dF", dF), ("lambda", lam)),
                                writable=("dY", "dF"))
    st = _stream_of(gy) if stream is None else _stream_handle(stream)
    _raise(L_.load().ffcm_adjoint(config.handle, gy.ptr, gf.ptr, l_.ptr, gy.memory, st))
    return dY, dF


def objective_gradient(config: FFCMConfig, Y, F, V_target, *, V=None, dY=None, dF=None, stream=None):
    """J = 0.5 |M(Y) F - V_target|^2 with its gradients, in one call.

    Returns ``(J, dJ/dY, dJ/dF, V)``. Host arrays give a float J; CUDA tensors
    give J as a one-element float64 CUDA tensor (the call stays asynchronous).
    """
    T = config.T
    dev = _is_torch(Y) and Y.is_cuda
    if dev:
        import torch
        mk = lambda: torch.empty_like(Y)  # noqa: E731
        Jbuf = torch.zeros(1, dtype=torch.float64, device=Y.device)
        jptr = ctypes.cast(ctypes.c_void_p(Jbuf.data_ptr()), ctypes.POINTER(ctypes.c_double))
    else:
        mk = lambda: np.empty((config.N, 3), T)  # noqa: E731
        Jbuf = ctypes.c_double(0.0)
        jptr = ctypes.pointer(Jbuf)
    V = mk() if V is None else V
    dY = mk() if dY is None else dY
    dF = mk() if dF is None else dF
    gy, gf, v, y, f, t = _particle_args(
        config, (("dY", dY), ("dF", dF), ("V", V), ("Y", Y), ("F", F), ("V_target", V_target)),
        writable=("dY", "dF", "V"))
    st = _stream_of(v) if stream is None else _stream_handle(stream)
    _raise(L_.load().ffcm_objective_gradient(config.handle, jptr, gy.ptr, gf.ptr, v.ptr, y.ptr, f.ptr,
                                             t.ptr, v.memory, st))
    return (Jbuf if dev else Jbuf.value), dY, dF, V


def rrule_mobility(config: FFCMConfig, Y, F):
    """Counterpart of a ChainRulesCore ``rrule`` for ``V = mobility(config, Y, F)``:
    returns ``(V, pullback)`` with ``pullback(Vbar) -> (Ybar, Fbar)``.

    The pullback is valid until the next solve on ``config``.
    """
    dev = _is_torch(Y) and Y.is_cuda
    if dev:
        import torch
        mk = lambda: torch.empty_like(Y)  # noqa: E731
    else:
        mk = lambda: np.empty((config.N, 3), config.T)  # noqa: E731
    V = mobility_checkpoint(mk(), config, Y, F)

    def pullback(Vbar):
        dY, dF = mk(), mk()
        adjoint(dY, dF, config, Vbar)
        return dY, dF

    return V, pullback


def _torch_function():
    import torch

    class MobilityFunction(torch.autograd.Function):
        """``V = M(Y) F`` on CUDA tensors with the hand-written pullback."""

        @staticmethod
        def forward(ctx, Y, F, config):
            V = torch.empty_like(Y)
            mobility_checkpoint(V, config, Y.detach().contiguous(), F.detach().contiguous())
            ctx.config = config
            return V

        @staticmethod
        def backward(ctx, Vbar):
            dY = torch.empty_like(Vbar)
            dF = torch.empty_like(Vbar)
            adjoint(dY, dF, ctx.config, Vbar.contiguous())
            return dY, dF, None

    return MobilityFunction


def mobility_autograd(config: FFCMConfig, Y, F):
    """Differentiable ``V = M(Y) F`` for CUDA tensors (torch.autograd)."""
    return _torch_function().apply(Y, F, config)


def validate_config(T, *, L, R_c, N, a=1.0, kernel_widths_ratio, num_grid_points, M_G,
                    viscosity, fft_planning="measure", fft_threads=1):
    """Host-only validation (no device work): raises as FFCMConfig would."""
    if fft_planning not in L_.FFT_PLANNING:
        raise ArgumentError(f"fft_planning must be :estimate, :measure, or :patient; got "
                            f":{fft_planning}")
    _raise(L_.load().ffcm_validate_config(
        _dtype_code(T), _dptr(L), float(R_c), int(N), float(a), float(kernel_widths_ratio),
        _i32ptr(num_grid_points), int(M_G), float(viscosity), L_.FFT_PLANNING[fft_planning],
        int(fft_threads)))


def derive_scalars(T, *, L, R_c, a=1.0, kernel_widths_ratio, num_grid_points):
    """Host-only derived scalars (``_derive_scalars``), returned in precision T."""
    T_ = np.dtype(T).type
    nc = (ctypes.c_int32 * 3)()
    cs = (ctypes.c_double * 3)()
    ics = (ctypes.c_double * 3)()
    s, S, hh, ih = (ctypes.c_double() for _ in range(4))
    _raise(L_.load().ffcm_derive_scalars(
        _dtype_code(T), _dptr(L), float(R_c), float(a), float(kernel_widths_ratio),
        _i32ptr(num_grid_points), nc, cs, ics, ctypes.byref(s), ctypes.byref(S),
        ctypes.byref(hh), ctypes.byref(ih)))
    return dict(num_cells=tuple(int(v) for v in nc), cell_size=tuple(T_(v) for v in cs),
                inv_cell_size=tuple(T_(v) for v in ics), sigma=T_(s.value), Sigma=T_(S.value),
                h=T_(hh.value), inv_h=T_(ih.value))


def batch_offsets(Ns, nrhs):
    """Row offsets of the batched layout (``ffcm_batch_create``): system i's
    positions start at row ``yoff[i]`` of the ``(sum N, 3)`` position array,
    its right-hand side r at row ``fvoff[i] + r * N[i]`` of the
    ``(nrhs * sum N, 3)`` force and velocity arrays."""
    Ns = np.asarray(Ns, np.int64)
    yoff = np.concatenate([[0], np.cumsum(Ns)[:-1]]).astype(np.int64)
    return yoff, int(nrhs) * yoff


def pack_batch(T, Ys=None, Fs=None):
    """Flatten per-system positions [(N_i, 3)] and forces [[(N_i, 3)] * nrhs]
    into the batched layout (host arrays of type T)."""
    out = []
    if Ys is not None:
        out.append(np.ascontiguousarray(np.concatenate([np.asarray(y, T).reshape(-1, 3) for y in Ys]), T))
    if Fs is not None:
        out.append(np.ascontiguousarray(np.concatenate(
            [np.asarray(f, T).reshape(-1, 3) for fr in Fs for f in fr]), T))
    return out[0] if len(out) == 1 else tuple(out)


def unpack_batch(V, Ns, nrhs):
    """Split a batched velocity array into [[(N_i, 3)] * nrhs] per system (views)."""
    V = np.asarray(V)
    _, fvoff = batch_offsets(Ns, nrhs)
    return [[V[fvoff[i] + r * n: fvoff[i] + (r + 1) * n] for r in range(int(nrhs))]
            for i, n in enumerate(int(x) for x in Ns)]


class FFCMBatch:
    """Batched form: ``nsys`` independent suspensions, each with ``nrhs`` force
    right-hand sides, solved by one CUDA-graph launch per call.

    Equivalent to ``mobility(V[i][r], FFCMConfig(systems[i]...), Y[i], F[i][r])``
    for every system i and right-hand side r. ``systems`` is a list of dicts
    with ``L``, ``R_c``, ``N``, ``num_grid_points``; the kernel widths ratio,
    ``M_G``, viscosity and ``a`` are shared. Arrays are flat: system i's
    positions are rows ``yoff[i]:yoff[i]+N[i]`` of an ``(sum N, 3)`` array and
    its right-hand side r is rows ``fvoff[i] + r*N[i] : ... + N[i]`` of an
    ``(nrhs * sum N, 3)`` array (see ``pack``/``unpack``).
    """

    def __init__(self, T=np.float32, *, systems, kernel_widths_ratio, M_G, viscosity, nrhs=1,
                 a=1.0, device=0):
        self._b = None
        self.T = np.dtype(T).type
        dt = _dtype_code(T)
        n = len(systems)
        if n < 1:
            raise ArgumentError("a batch needs at least one system")
        Ls = [float(x) for s_ in systems for x in s_["L"]]
        Rc = [float(s_["R_c"]) for s_ in systems]
        Ns = [int(s_["N"]) for s_ in systems]
        Ms = [int(m) for s_ in systems for m in s_["num_grid_points"]]
        b = ctypes.c_void_p()
        _raise(L_.load().ffcm_batch_create(
            ctypes.byref(b), dt, n, _dptr(Ls), _dptr(Rc), (ctypes.c_int64 * n)(*Ns), float(a),
            float(kernel_widths_ratio), _i32ptr(Ms), int(M_G), float(viscosity), int(nrhs),
            int(device)))
        self._b = b
        self.device = int(device)
        self.N = Ns
        self.nrhs = int(nrhs)
        self.nsys = n
        self.yoff, self.fvoff = batch_offsets(Ns, self.nrhs)
        total, ns, nr, kern = (ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(),
                               ctypes.c_int64())
        _raise(L_.load().ffcm_batch_get_info(b, ctypes.byref(total), ctypes.byref(ns),
                                             ctypes.byref(nr), ctypes.byref(kern)))
        self.total_particles = int(total.value)
        self.kernels_per_call = int(kern.value)

    def close(self):
        if getattr(self, "_b", None):
            L_.load().ffcm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, Ys=None, Fs=None):
        """Flatten per-system positions [(N_i,3)] and forces [[(N_i,3)] * nrhs]."""
        return pack_batch(self.T, Ys, Fs)

    def unpack(self, V):
        """Split a flat velocity array into [[(N_i,3)] * nrhs] per system."""
        return unpack_batch(V, self.N, self.nrhs)

    def mobility(self, V, Y, F, stream=None):
        T = self.T
        tot = self.total_particles
        v = _Arg(V, T, writable=True, device=self.device)
        y = _Arg(Y, T, device=self.device)
        f = _Arg(F, T, device=self.device)
        if (y.rows, y.cols) != (3, tot) or (f.rows, f.cols) != (3, tot * self.nrhs) or \
                (v.rows, v.cols) != (3, tot * self.nrhs):
            raise DimensionMismatch("batch arrays must be (sum N, 3) for Y and "
                                    "(nrhs * sum N, 3) for F and V")
        if len({v.memory, y.memory, f.memory}) != 1:
            raise ArgumentError("V, Y and F must all be host arrays or all be CUDA tensors")
        st = _stream_of(v) if stream is None else _stream_handle(stream)
        _raise(L_.load().ffcm_batch_mobility(self._b, v.ptr, y.ptr, f.ptr, v.memory, st))
        return V


# ---- one system over several GPUs: z-slab decomposition (ffcm_dist_*) ----

def dist_partition(T, num_grid_points, nranks, rank):
    """``(z_begin, z_end, kx_begin, kx_end)`` of ``rank`` in a z-slab
    decomposition over ``nranks`` (host only: ``ffcm_dist_partition``)."""
    out = (ctypes.c_int32 * 4)()
    _raise(L_.load().ffcm_dist_partition(_dtype_code(T), _i32ptr(num_grid_points), int(nranks), int(rank), out))
    return tuple(int(v) for v in out)


class _DeviceArray:
    """A device buffer of the library seen by torch without a copy
    (``__cuda_array_interface__``)."""

    def __init__(self, ptr, count, typestr, device):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}
        self.device = device

    def tensor(self):
        import torch
        return torch.as_tensor(self, device=f"cuda:{self.device}")


class TorchExchange:
    """The collectives of a z-slab decomposition through torch.distributed:
    the two spectrum transposes as ``all_to_all_single`` of R equal blocks and
    the interpolation shares as an ``all_reduce`` (sum). With the NCCL backend
    the tensors stay on the GPU."""

    def __init__(self, group=None):
        self.group = group

    def all_to_all(self, recv, send):
        import torch.distributed as dist
        dist.all_to_all_single(recv, send, group=self.group)

    def all_reduce(self, partial):
        import torch.distributed as dist
        dist.all_reduce(partial, op=dist.ReduceOp.SUM, group=self.group)


class LocalExchange:
    """The collectives of a decomposition over one rank: the transposes are
    copies and the sum is the identity."""

    def all_to_all(self, recv, send):
        recv.copy_(send)

    def all_reduce(self, partial):
        pass


class DistributedConfig:
    """One rank of a configuration split over ``nranks`` GPUs by z slabs
    (``ffcm_dist_create``): the same parameters as ``FFCMConfig``, the grid
    divided so that each GPU holds 1 / nranks of the spectrum. The particles
    are replicated. ``mobility(V, Y, F, exchange)`` runs the steps of
    ``ffcm_dist_*`` with the exchange's collectives between them; every rank
    receives all N velocities. No reference counterpart (the reference solves
    one system per device)."""

    def __init__(self, T=np.float32, *, rank, nranks, L, R_c, N, a=1.0, kernel_widths_ratio, num_grid_points,
                 M_G, viscosity, device=0, stencil=None, **_ignored):
        self._h = None
        self.T = np.dtype(T).type
        self.rank, self.nranks, self.device, self.N = int(rank), int(nranks), int(device), int(N)
        lib = L_.load()
        h = ctypes.c_void_p()
        _raise(lib.ffcm_dist_create(ctypes.byref(h), _dtype_code(T), _dptr(L), float(R_c), int(N), float(a),
                                    float(kernel_widths_ratio), _i32ptr(num_grid_points), int(M_G),
                                    float(viscosity), int(nranks), int(rank), int(device)))
        self._h = h
        if stencil is not None:
            _raise(lib.ffcm_set_stencil(h, L_.STENCIL[stencil]))
        send, recv, part = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        blk = ctypes.c_int64()
        rng = (ctypes.c_int32 * 4)()
        _raise(lib.ffcm_dist_buffers(h, ctypes.byref(send), ctypes.byref(recv), ctypes.byref(blk),
                                     ctypes.byref(part), rng))
        self.ranges = tuple(int(v) for v in rng)
        tstr = "<f4" if self.T == np.float32 else "<f8"
        words = int(blk.value) // np.dtype(self.T).itemsize * int(nranks)
        self.send = _DeviceArray(send.value, words, tstr, self.device).tensor()
        self.recv = _DeviceArray(recv.value, words, tstr, self.device).tensor()
        self.partial = _DeviceArray(part.value, 3 * self.N, tstr, self.device).tensor()

    def close(self):
        if getattr(self, "_h", None):
            L_.load().ffcm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if not self._h:
            raise FFCMError("configuration is closed")
        return self._h

    profile_begin = FFCMConfig.profile_begin
    profile_end = FFCMConfig.profile_end
    tuning = FFCMConfig.tuning
    launch_count = FFCMConfig.launch_count

    # the steps, on the current torch stream
    def _stream(self):
        import torch
        return _stream_handle(torch.cuda.current_stream(self.device))

    def forward(self, Y, F):
        y, f = _particle_args(self, (("Y", Y), ("F", F)))
        _raise(L_.load().ffcm_dist_forward(self._h, y.ptr, f.ptr, y.memory,
                                           self._stream() if y.memory == L_.DEVICE else None))

    def stokes(self):
        _raise(L_.load().ffcm_dist_stokes(self._h, self._stream()))

    def interpolate(self):
        _raise(L_.load().ffcm_dist_interpolate(self._h, self._stream()))

    def correct(self, V):
        (v,) = _particle_args(self, (("V", V),), writable=("V",))
        _raise(L_.load().ffcm_dist_correct(self._h, v.ptr, v.memory,
                                           self._stream() if v.memory == L_.DEVICE else None))
        return V

    def mobility(self, V, Y, F, exchange):
        """V = M(Y) F for the whole system, this rank's share of the work and
        the exchange's collectives in between."""
        self.forward(Y, F)
        exchange.all_to_all(self.recv, self.send)
        self.stokes()
        exchange.all_to_all(self.recv, self.send)
        self.interpolate()
        exchange.all_reduce(self.partial)
        return self.correct(V)


def distributed_mobility_local(configs, Vs, Y, F):
    """All ranks of a decomposition driven from one process (one GPU or
    several): the collectives become copies between the ranks' buffers, in
    the order the processes of a real run would perform them. ``Vs`` holds
    one output array per rank."""
    import torch
    R = len(configs)
    for c in configs:
        c.forward(Y, F)

    def exchange():
        blocks = [c.send.view(R, -1).clone() for c in configs]
        for r, c in enumerate(configs):
            for q in range(R):
                c.recv.view(R, -1)[q].copy_(blocks[q][r])

    for c in configs:
        torch.cuda.current_stream(c.device).synchronize()
    exchange()
    for c in configs:
        c.stokes()
    for c in configs:
        torch.cuda.current_stream(c.device).synchronize()
    exchange()
    for c in configs:
        c.interpolate()
    for c in configs:
        torch.cuda.current_stream(c.device).synchronize()
    total = sum(c.partial.clone() for c in configs)
    for c in configs:
        c.partial.copy_(total)
    for c, V in zip(configs, Vs):
        c.correct(V)
    return Vs
