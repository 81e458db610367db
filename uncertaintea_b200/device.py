"""``UncertainTea.Device`` mirror: batched logjoint / gradient on the B200.

reference facade: src/UncertainTea.jl:189-200; entry points
src/device/api.jl:18 (device_batched_logjoint), :55
(device_batched_logjoint_gradient), :82 (the workspace-reuse `!` form),
src/device/workspace.jl:71 (DeviceBatchedWorkspace) and :24-35
(device_lowering_report / the unsupported-model message).

Host-array calls take and return numpy arrays laid out like the reference:
``params`` is P x C (rows = unconstrained parameters, columns = chains).
Device calls take torch CUDA tensors of shape (C, P), which is the same
memory layout as the reference's column-major P x C matrix.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat
from .models import TeaModelSpec


def _check_precision(precision):
    if precision is None:
        return
    if precision in (np.float32, "float32", "Float32") or getattr(precision, "__name__", "") == "float32":
        return
    try:
        import torch
        if precision is torch.float32:
            return
    except ImportError:  # pragma: no cover
        pass
    raise ValueError(
        f"backend cuda does not support {precision} arithmetic; request precision=Float32 instead")


def _torch():
    import torch
    return torch


def _resolve_device(backend):
    torch = _torch()
    if backend is None:
        raise ValueError("a device backend is required (e.g. backend='cuda'); the B200 path has no CPU fallback")
    dev = torch.device(backend) if not isinstance(backend, torch.device) else backend
    if dev.type != "cuda":
        raise ValueError(f"backend must be a CUDA device, got {dev}")
    return dev


def _stream_handle():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _host_output(shape):
    """A fresh float32 host array in page-locked memory for a device->host result.

    Drawn from torch's caching pinned-host allocator: after the first call a block
    of the same size is reused without registering pages again, and the copy runs
    at DMA speed without first-touch page faults or a staging bounce.  The array
    owns its block (through the tensor it views) until it is dropped, so each call
    returns independent arrays, as the reference's allocating copies do
    (src/device/api.jl:103-106).  The library's own copy is synchronised before
    the entry point returns, so a block freed later has no copy in flight."""
    torch = _torch()
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def device_lowering_report(model: TeaModelSpec, args=(), constraints=None):
    """(supported, issues) for a model's kernel description (workspace.jl:24-35)."""
    lib = nat.load()
    try:
        lowered = model.lower(args, constraints)
    except (ValueError, IndexError) as err:
        return False, [str(err)]
    buf = ctypes.create_string_buffer(4096)
    prog = getattr(lowered, "program", None)
    if prog is not None:
        status = lib.ut_program_report(lowered.steps, len(prog.steps), lowered.nodes, len(prog.nodes), prog.num_slots,
                                       prog.num_params, int(lowered.observed.size), buf, len(buf))
    else:
        status = lib.ut_lowering_report(ctypes.byref(lowered.plan), buf, len(buf))
    issues = [s for s in buf.value.decode().split("\n") if s]
    return status == nat.UT_OK, issues


class DeviceBatchedWorkspace:
    """Device-resident workspace (src/device/workspace.jl:37-137): the lowered
    kernel description, the staged observations and the reusable buffers of
    one batch of ``num_chains`` chains."""

    def __init__(self, model: TeaModelSpec, num_chains: int, *, backend="cuda", precision=None, args=(),
                 constraints=None):
        _check_precision(precision)
        self.lib = nat.load()
        self.model = model
        self.args = args
        self.constraints = constraints
        self.device = _resolve_device(backend)
        torch = _torch()
        if self.device.index is not None:
            torch.cuda.set_device(self.device)
        lowered = model.lower(args, constraints)
        self.lowered = lowered
        handle = ctypes.c_void_p()
        obs = lowered.observed
        prog = getattr(lowered, "program", None)
        if prog is not None:
            status = self.lib.ut_workspace_create_program(
                lowered.steps, len(prog.steps), lowered.nodes, len(prog.nodes), prog.num_slots, prog.num_params,
                nat.ptr(obs) if obs.size else None, int(obs.size), int(num_chains), 32, ctypes.byref(handle))
        else:
            status = self.lib.ut_workspace_create(
                ctypes.byref(lowered.plan), nat.ptr(obs), int(obs.size), 1,
                nat.ptr(lowered.trip_counts) if lowered.trip_counts.size else None,
                nat.ptr(lowered.loop_starts) if lowered.loop_starts.size else None,
                int(lowered.trip_counts.size), int(num_chains), 32, ctypes.byref(handle))
        if status == nat.UT_ERR_UNSUPPORTED:
            msg = nat.last_error()
            raise ValueError(f"model {model.name} cannot be lowered to the device logjoint path. Issues:\n  - "
                             + msg.split("\n", 1)[-1].replace("\n", "\n  - ")
                             + "\nSee device_lowering_report(model) for details.")
        nat.check(status)
        self.handle = handle
        self.parameter_count = lowered.num_params
        self.batch_size = int(num_chains)

    def kernel_path(self) -> str:
        """'warp' (one warp per chain), 'tiled' (CUDA-core GEMM tiles), 'tensor_core' (tcgen05 3xTF32) or
        'stream' (few chains: the HBM-streaming kernel)."""
        return {1: "warp", 2: "tiled", 3: "tensor_core", 4: "stream"}.get(self.lib.ut_workspace_path(self.handle),
                                                                             "unknown")

    def tensor_core_path(self) -> bool:
        return self.kernel_path() == "tensor_core"

    def launches_per_gradient(self) -> int:
        """Kernels one logjoint+gradient call launches (the bench's launch count)."""
        return {"warp": 1, "tiled": 2, "tensor_core": 3, "stream": 1}[self.kernel_path()]

    def check(self):
        """Synchronise and raise if a bounded in-kernel wait gave up."""
        nat.check(self.lib.ut_workspace_check(self.handle, _stream_handle()))

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.ut_workspace_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- shape checks mirroring src/device/api.jl:83-93 ----------------------
    def _check_host_params(self, params):
        params = np.asarray(params)
        if params.ndim != 2 or params.shape[0] != self.parameter_count:
            raise IndexError(f"expected {self.parameter_count} unconstrained parameters (rows), got "
                             f"{params.shape[0] if params.ndim == 2 else params.shape}")
        if params.shape[1] != self.batch_size:
            raise IndexError(f"expected {self.batch_size} batch elements, got {params.shape[1]}")
        # P x C (reference layout) -> chain-major contiguous float32.  A P x C view of
        # chain-major float32 memory is passed as it is; otherwise the converted copy
        # is written into page-locked memory, so the upload needs no staging bounce.
        qt = params.T
        if qt.dtype == np.float32 and qt.flags.c_contiguous:
            return qt
        q = _host_output(qt.shape)
        np.copyto(q, qt, casting="unsafe")
        return q

    def _check_device_params(self, params):
        torch = _torch()
        if not isinstance(params, torch.Tensor) or not params.is_cuda:
            raise ValueError("device calls take CUDA tensors")
        if params.dtype != torch.float32:
            raise ValueError(f"expected float32 parameters, got {params.dtype}")
        if tuple(params.shape) != (self.batch_size, self.parameter_count):
            raise IndexError(f"expected a ({self.batch_size}, {self.parameter_count}) chain-major tensor, "
                             f"got {tuple(params.shape)}")
        return params.contiguous()

    # -- host-array entry points (copy in, compute, copy out) -----------------
    def logjoint(self, params) -> np.ndarray:
        """device_batched_logjoint!(ws, params) -> Vector (C,)."""
        q = self._check_host_params(params)
        totals = _host_output(self.batch_size)
        nat.check(self.lib.ut_logjoint(self.handle, nat.ptr(q), nat.ptr(totals)))
        return totals

    def logjoint_gradient(self, params):
        """device_batched_logjoint_gradient!(ws, params) -> (values (C,), gradients (P, C))."""
        q = self._check_host_params(params)
        totals = _host_output(self.batch_size)
        grads = _host_output((self.batch_size, self.parameter_count))
        nat.check(self.lib.ut_logjoint_gradient(self.handle, nat.ptr(q), nat.ptr(totals), nat.ptr(grads)))
        return totals, grads.T

    # -- device-tensor entry points ------------------------------------------
    def logjoint_device(self, params, totals=None):
        torch = _torch()
        params = self._check_device_params(params)
        if totals is None:
            totals = torch.empty(self.batch_size, dtype=torch.float32, device=params.device)
        nat.check(self.lib.ut_logjoint_device(self.handle, nat.ptr(params), nat.ptr(totals), _stream_handle()))
        return totals

    def logjoint_gradient_device(self, params, totals=None, gradients=None):
        torch = _torch()
        params = self._check_device_params(params)
        if totals is None:
            totals = torch.empty(self.batch_size, dtype=torch.float32, device=params.device)
        if gradients is None:
            gradients = torch.empty_like(params)
        nat.check(self.lib.ut_logjoint_gradient_device(self.handle, nat.ptr(params), nat.ptr(totals),
                                                       nat.ptr(gradients), _stream_handle()))
        return totals, gradients


def device_batched_logjoint(model, params, args=(), constraints=None, *, backend="cuda", precision=None):
    """Batched unconstrained logjoint of every column of ``params`` (P x C)."""
    params = np.asarray(params)
    ws = DeviceBatchedWorkspace(model, params.shape[1] if params.ndim == 2 else 1, backend=backend,
                                precision=precision, args=args, constraints=constraints)
    try:
        return ws.logjoint(params)
    finally:
        ws.close()


def device_batched_logjoint_gradient(model, params, args=(), constraints=None, *, backend="cuda", precision=None):
    """Batched logjoint and gradient: (values (C,), gradients (P, C))."""
    params = np.asarray(params)
    ws = DeviceBatchedWorkspace(model, params.shape[1] if params.ndim == 2 else 1, backend=backend,
                                precision=precision, args=args, constraints=constraints)
    try:
        return ws.logjoint_gradient(params)
    finally:
        ws.close()


def device_batched_logjoint_(ws: DeviceBatchedWorkspace, params):
    """Workspace-reuse form (the reference's ``device_batched_logjoint!``)."""
    return ws.logjoint(params)


def device_batched_logjoint_gradient_(ws: DeviceBatchedWorkspace, params):
    """Workspace-reuse form (the reference's ``device_batched_logjoint_gradient!``)."""
    return ws.logjoint_gradient(params)
