"""Many circuits of different qubit counts evaluated as one unit: one CUDA-graph launch per call.

``CircuitBatch`` takes members (n_qubits, circuit, Hamiltonians) that do not share a register
size, so they cannot share one batched launch of the tile kernels.  It allocates every state,
workspace and output once, picks each member's tile width (fusion width) by timing candidate
widths on the device (``autotune``), and records the launches of all members (forward passes,
Hamiltonian, adjoint sweep, gradient scatter) into one CUDA graph whose members run on several
streams, so small registers that cannot fill the GPU alone run side by side.  A call copies the
parameters into the graph's input buffers, replays the graph and returns every member's
expectations and gradients.  This is the batched counterpart of calling
``get_expectation_with_grad`` once per circuit (mindquantum/simulator/mqsim.py:255-439).
"""
import ctypes
import math

import numpy as np
import torch

from .. import _native as N
from ..dtype import complex64, complex128
from .lowering import Program, native_ham


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


class _Member:
    def __init__(self, n, circuit, hams, precision, device):
        self.n = n
        self.circuit = circuit
        self.hams = [hams] if not isinstance(hams, (list, tuple)) else list(hams)
        self.names = list(circuit.params_name)
        self.nh = [native_ham(h, n, precision) for h in self.hams]
        self.ham_arr = (ctypes.c_void_p * len(self.nh))(*[h.handle.value for h in self.nh])
        self.precision = precision
        self.device = device
        self.params = torch.zeros((1, max(1, len(self.names))), dtype=torch.float64, device=device)
        self.f = torch.zeros((1, len(self.nh), 2), dtype=torch.float64, device=device)
        self.g = torch.zeros((1, len(self.nh), max(1, len(self.names))), dtype=torch.float64, device=device)
        self.prog = None
        self.tile_bits = 0
        self.stride = 1
        self.ws = None

    def program(self, tile_bits):
        return Program(self.circuit, self.n, self.precision, self.names, None, True, tile_bits)

    def workspace_bytes(self, prog, stride):
        ws = ctypes.c_size_t()
        N.call('mqb_grad_workspace_size', prog.handle, 1, len(self.nh), stride, ctypes.byref(ws))
        return ws.value

    def launch(self, prog, ws, stride, stream):
        N.call('mqb_expectation_with_grad', prog.handle, self.ham_arr, len(self.nh), None, 0, 1, _ptr(self.params),
               self.params.shape[1], None, _ptr(self.f), _ptr(self.g), stride, _ptr(ws), ws.numel(),
               ctypes.c_void_p(stream.cuda_stream))


class CircuitBatch:
    """Expectations and adjoint gradients of many independent circuits per call.

    Args:
        members: list of ``(n_qubits, circuit, hamiltonian_or_list)``; circuits without
            measurements, every parameter gets a gradient.
        dtype: ``complex64`` (FP32 states, FP64 reductions) or ``complex128``.
        autotune: pick each member's tile width by timing (else the library default).
        graph: record all launches into one CUDA graph (else launch member by member).
        streams: streams the members are spread over inside the graph.
        memory_fraction: share of the free device memory the workspaces may take; members whose
            checkpoints do not fit recompute states (checkpoint every sqrt(passes) passes, or none).
    """

    def __init__(self, members, dtype=complex64, autotune=True, graph=True, streams=8, memory_fraction=0.7):
        if not torch.cuda.is_available():
            raise RuntimeError("CircuitBatch needs a CUDA device (B200, sm_100a); none is visible")
        self.device = torch.device('cuda', torch.cuda.current_device())
        self.precision = N.MQB_PREC_C64 if dtype == complex64 else N.MQB_PREC_C128
        if dtype not in (complex64, complex128):
            raise TypeError(f"dtype must be complex64 or complex128, got {dtype}")
        self.members = [_Member(n, c, h, self.precision, self.device) for n, c, h in members]
        self._pack()
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, min(streams, len(self.members))))]
        self._plan(autotune, memory_fraction)
        self.graph = None
        if graph:
            self._capture()

    def _pack(self):
        """Every member's parameters, expectations and gradients as views into three device
        buffers (the graph records the views' addresses), with pinned host mirrors: a call moves
        the whole batch's inputs and outputs with one copy per buffer."""
        n_p = [m.params.numel() for m in self.members]
        n_f = [m.f.numel() for m in self.members]
        n_g = [m.g.numel() for m in self.members]
        self._p_off, self._f_off, self._g_off = (np.concatenate([[0], np.cumsum(x)]).astype(np.int64)
                                                 for x in (n_p, n_f, n_g))
        self.params_all = torch.zeros(int(self._p_off[-1]), dtype=torch.float64, device=self.device)
        self.f_all = torch.zeros(int(self._f_off[-1]), dtype=torch.float64, device=self.device)
        self.g_all = torch.zeros(int(self._g_off[-1]), dtype=torch.float64, device=self.device)
        for i, m in enumerate(self.members):
            m.params = self.params_all[self._p_off[i]:self._p_off[i + 1]].view(m.params.shape)
            m.f = self.f_all[self._f_off[i]:self._f_off[i + 1]].view(m.f.shape)
            m.g = self.g_all[self._g_off[i]:self._g_off[i + 1]].view(m.g.shape)
        self._p_host = torch.zeros(self.params_all.numel(), dtype=torch.float64, pin_memory=True)
        self._f_host = torch.zeros(self.f_all.numel(), dtype=torch.float64, pin_memory=True)
        self._g_host = torch.zeros(self.g_all.numel(), dtype=torch.float64, pin_memory=True)

    # ------------------------------------------------------------------------------ planning
    def _plan(self, autotune, memory_fraction):
        free, _ = torch.cuda.mem_get_info(self.device)
        budget = memory_fraction * free
        # strides: every pass stored while the total fits, largest members recompute first
        for m in self.members:
            m.prog = m.program(0)
            m.stride = 1
        order = sorted(range(len(self.members)), key=lambda i: -self.members[i].n)

        def total():
            return sum(m.workspace_bytes(m.prog, m.stride) for m in self.members)

        for i in order:
            if total() <= budget:
                break
            m = self.members[i]
            passes = m.prog.grad_passes(len(m.nh))[0]
            m.stride = max(2, int(math.ceil(math.sqrt(max(1, passes)))))
            if total() > budget:
                m.stride = 0
        if total() > budget:
            raise MemoryError("the batch's states do not fit in device memory")
        for m in self.members:
            m.ws = torch.empty(max(256, m.workspace_bytes(m.prog, m.stride)), dtype=torch.uint8, device=self.device)
        if autotune:
            for m in self.members:
                self._tune(m)

    def _tune(self, m):
        """Time the member's gradient at candidate tile widths; keep the fastest (ties: default).

        Members of 18 qubits and more run generated pass kernels, whose compile time per candidate
        would dominate; they keep the default width.
        """
        k0 = m.prog.info.tile_bits
        cands = [0] if m.n >= 18 else sorted({0, *[k for k in (k0 - 2, k0 - 1, k0 + 1) if 6 <= k <= 13 and k <= m.n]})
        best = None
        stream = self.streams[0]
        for k in cands:
            prog = m.prog if k == 0 else m.program(k)
            need = m.workspace_bytes(prog, m.stride)
            if need > m.ws.numel():
                continue
            with torch.cuda.stream(stream):
                m.params.uniform_(0, 2 * np.pi)
                m.launch(prog, m.ws, m.stride, stream)   # warm-up
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0.record(stream)
                for _ in range(3):
                    m.launch(prog, m.ws, m.stride, stream)
                t1.record(stream)
            t1.synchronize()
            ms = t0.elapsed_time(t1) / 3
            if best is None or ms < best[0] * 0.97:
                best = (ms, k, prog)
        m.tile_bits, m.prog = best[1], best[2]
        m.tuned_ms = best[0]

    # ------------------------------------------------------------------------------ execution
    def _launch_all(self, main):
        done = []
        for i, m in enumerate(self.members):
            s = self.streams[i % len(self.streams)]
            if i < len(self.streams):
                s.wait_stream(main)
            m.launch(m.prog, m.ws, m.stride, s)
        for s in self.streams:
            main.wait_stream(s)
            done.append(s)
        return done

    def _capture(self):
        torch.cuda.synchronize(self.device)
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=self.device)
        with torch.cuda.graph(self.graph, stream=side):
            self._launch_all(torch.cuda.current_stream())
        torch.cuda.synchronize(self.device)

    def __call__(self, params_list):
        """Expectations f[i] ([n_hams] complex) and gradients g[i] ([n_hams][n_params]) of every member."""
        if len(params_list) != len(self.members):
            raise ValueError(f"expected {len(self.members)} parameter vectors, got {len(params_list)}")
        for m, p in zip(self.members, params_list):
            p = torch.as_tensor(p, dtype=torch.float64).reshape(-1)
            if p.numel() != len(m.names):
                raise ValueError(f"member with {len(m.names)} parameters got {p.numel()} values")
            if p.numel():
                m.params[0, :p.numel()].copy_(p, non_blocking=True)
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch_all(torch.cuda.current_stream())
        out_f, out_g = [], []
        for m in self.members:
            f = m.f[0]
            out_f.append(torch.complex(f[:, 0], f[:, 1]))
            out_g.append(m.g[0, :, :len(m.names)])
        return out_f, out_g

    def evaluate(self, params_list):
        """Host in, host out: every member's parameters gathered into one pinned buffer and copied
        with one host-to-device copy, one replay, and the expectations and gradients of all members
        read back with one device-to-host copy per buffer.  Returns (f, g): lists of numpy arrays,
        f[i] [n_hams] complex, g[i] [n_hams][n_params]."""
        if len(params_list) != len(self.members):
            raise ValueError(f"expected {len(self.members)} parameter vectors, got {len(params_list)}")
        host = self._p_host.numpy()
        for i, (m, p) in enumerate(zip(self.members, params_list)):
            p = np.asarray(p, dtype=np.float64).reshape(-1)
            if p.size != len(m.names):
                raise ValueError(f"member with {len(m.names)} parameters got {p.size} values")
            host[self._p_off[i]:self._p_off[i] + p.size] = p
        self.params_all.copy_(self._p_host, non_blocking=True)
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch_all(torch.cuda.current_stream())
        self._f_host.copy_(self.f_all, non_blocking=True)
        self._g_host.copy_(self.g_all, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        fh, gh = self._f_host.numpy(), self._g_host.numpy()
        out_f, out_g = [], []
        for i, m in enumerate(self.members):
            f = fh[self._f_off[i]:self._f_off[i + 1]].reshape(len(m.nh), 2)
            out_f.append(f[:, 0] + 1j * f[:, 1])
            g = gh[self._g_off[i]:self._g_off[i + 1]].reshape(len(m.nh), -1)
            out_g.append(g[:, :len(m.names)].copy())
        return out_f, out_g

    def launches_per_call(self):
        """Kernel launches recorded in the graph (one replay launches them all)."""
        with N.KernelTimer() as kt:
            self._launch_all(torch.cuda.current_stream())
            torch.cuda.synchronize(self.device)
        return sum(kt.launches.values())
