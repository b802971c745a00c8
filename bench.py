"""Benchmark: batched complex64 adjoint gradients of a 26-qubit hardware-efficient ansatz on B200.

Workload (one "step" = one batched gradient evaluation): 26 qubits, 12 layers of RY then RZ on
every qubit followed by a CNOT ladder q_i -> q_{i+1} (624 parameters, 924 gates); the
Hamiltonian H = sum_i a_i Z_i Z_{i+1} + sum_i b_i X_i (51 terms, a, b ~ N(0, 1)); a batch of B
parameter sets (encoder samples) with angles ~ U[0, 2pi).  Every step computes <H> and the full
624-entry gradient for every sample, complex64 state with FP64 reductions.  Synthetic data from
numpy.random.default_rng(0): angles first, then Hamiltonian coefficients.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank runs its own batch (replicas, weak scaling, no data-path collective);
the timed region is bracketed by a barrier and a device synchronize and the max over ranks is
reported.  ``--impl reference`` times the reference's own CPU simulator (built from its sources into
oracle/_ref; the oracle port of its kernels where that is not built) on the host cores: full
gradient evaluations of the workload, at most three (a bounded run).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault('MQB_JIT_CACHE', os.path.join(ROOT, '_build', 'jit_cache'))
METRIC = "grad evals/s at 26q c64-batched vs c128-plain, same B200, err≤1e-5; HBM GB/s"
UNIT = "grad evals/s"


def build_workload(n, layers, batch, seed=0):
    from mindquantum_b200.core import gates as G
    from mindquantum_b200.core.circuit import Circuit
    from mindquantum_b200.core.operators import Hamiltonian, QubitOperator

    circ = Circuit()
    k = 0
    for _ in range(layers):
        for q in range(n):
            circ += G.RY(f'p{k}').on(q)
            k += 1
        for q in range(n):
            circ += G.RZ(f'p{k}').on(q)
            k += 1
        for q in range(n - 1):
            circ += G.X.on(q + 1, q)
    circ.as_encoder()
    rng = np.random.default_rng(seed)
    params = rng.uniform(0, 2 * np.pi, size=(batch, k))
    a = rng.normal(size=n - 1)
    b = rng.normal(size=n)
    op = QubitOperator()
    for i in range(n - 1):
        op += QubitOperator(f'Z{i} Z{i + 1}', float(a[i]))
    for i in range(n):
        op += QubitOperator(f'X{i}', float(b[i]))
    return circ, Hamiltonian(op), params


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.QUERY}', '--format=csv,noheader,nounits',
                                          '-i', str(self.gpu), '-lms', '200'], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(',')])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == 'active':
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json'), encoding='utf8') as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


# DRAM bytes per state byte moved by one adjoint pass launch (psi read, lambda read + write: 3 x
# S*B algorithmic), from an ncu capture of the same kernel on the HEA 24-qubit, batch-2 case; a
# launch's traffic grows in proportion to the state bytes it processes (760.9 and 761.6 MB read +
# written for S*B = 268.4 MB in the two captured launches).  None: not captured for
# the kernels built from the current sources.
ADJ_DRAM_BYTES_PER_STATE_BYTE = 2.84


def oracle_fixture_errors(n, layers, batch, seed, f_c64, g_c64, f_c128=None, g_c128=None):
    """max |delta| of <H> and the gradient of parameter set 0 against the FP64 oracle's result for the
    same workload (tests/golden/hea26_oracle.json, made by tests/golden/make_oracle_fixtures.py)."""
    path = os.path.join(ROOT, 'tests', 'golden', f'hea{n}_oracle.json')
    if seed != 0 or not os.path.exists(path):
        return {}
    with open(path, encoding='utf8') as f:
        fx = json.load(f)
    if fx.get('layers') != layers or fx.get('batch') != batch:
        return {}
    row = fx['samples'][0]
    ref_g = np.array(row['grad'])
    out = {"oracle_fixture": os.path.relpath(path, ROOT),
           "f_err_vs_oracle_c64": abs(float(f_c64) - row['f']),
           "grad_err_vs_oracle_c64": float(np.max(np.abs(np.asarray(g_c64) - ref_g)))}
    if g_c128 is not None:
        out["f_err_vs_oracle_c128"] = abs(float(f_c128) - row['f'])
        out["grad_err_vs_oracle_c128"] = float(np.max(np.abs(np.asarray(g_c128) - ref_g)))
    return out


def apply_throughput(sim, circ, names, params, n, B, reps, peak):
    """Fused gate application alone: the circuit applied in place to B resident states (mqb_apply,
    one generated kernel per pass), gates/s and the HBM fraction of its passes."""
    import torch

    from mindquantum_b200 import _native as N
    from mindquantum_b200.simulator import lowering

    prog = lowering.lowered(circ, n, sim.precision, names, None, True)
    states = torch.zeros((B, 1 << n), dtype=sim.torch_dtype, device=sim.device)
    states[:, 0] = 1
    ws_b = ctypes.c_size_t()
    N.call('mqb_apply_workspace_size', prog.handle, B, ctypes.byref(ws_b))
    ws = torch.empty(max(256, ws_b.value), dtype=torch.uint8, device=sim.device)
    st = torch.cuda.current_stream()

    def run():
        N.call('mqb_apply', prog.handle, ctypes.c_void_p(states.data_ptr()), B, ctypes.c_void_p(params.data_ptr()),
               params.shape[1], None, ctypes.c_void_p(ws.data_ptr()), ws_b.value, ctypes.c_void_p(st.cuda_stream))

    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        run()
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    S = (1 << n) * states.element_size() * B
    passes = prog.info.n_passes
    alg = 2 * S * passes
    del states, ws
    return {"gates_per_s": len(circ) * B / (ms / 1e3), "ms_per_apply": ms, "gates": len(circ), "states": B,
            "passes": passes, "tile_bits": prog.info.tile_bits, "alg_bytes": alg,
            "achieved_gbs": alg / (ms / 1e3) / 1e9, "frac": alg / (ms / 1e3) / 1e9 / peak,
            "bytes_model": "passes x 2 x S x B (every pass reads and writes each state once)"}


def reference_full_evaluations(n, layers, batch, threads, count):
    """Time full gradient evaluations of the workload on the host: the reference's own CPU
    simulator (VectorState<CPUVectorPolicyAvxFloat>, built from the reference sources into
    oracle/_ref), or the oracle port of its kernels where that library was not built.  One
    evaluation = <H> and the full gradient of parameter set 0 (all layers, the real lambda = H psi),
    complex64 like the benchmark.  Returns (seconds per evaluation list, kind)."""
    from oracle import refbin as R

    circ, ham, params = build_workload(n, layers, batch)
    times = []
    if R.available():
        kind = "reference"
        for _ in range(count):
            t0 = time.perf_counter()
            R.grad(n, circ, ham, params[:1], threads=threads, complex64=True)
            times.append(time.perf_counter() - t0)
    else:
        from oracle import oracle as O

        kind = "port"
        O.set_num_threads(threads)
        for _ in range(count):
            t0 = time.perf_counter()
            O.get_expectation_with_grad(n, [ham], circ, params[:1], np.zeros(0), circ.params_name, [], np.complex64)
            times.append(time.perf_counter() - t0)
    return times, kind


def reference_gpu_evaluations(args, count, warmup):
    """Seconds per full gradient evaluation of parameter set 0 on the reference's own thrust GPU
    simulator (`mqvector_gpu`, built from its sources for sm_100a into oracle/_ref/libmqref_gpu.so),
    one evaluation at a time as the reference runs them: {"c64": [...], "c128": [...]}.  Its API is
    synchronous and returns host values, so each evaluation is timed on the host clock between
    device synchronizations."""
    import torch

    from oracle import refbin as R

    circ, ham, params = build_workload(args.qubits, args.layers, args.batch)
    c1, h1, p1 = build_workload(args.qubits, 1, args.batch)
    out = {}
    for prec, c64 in (("c64", True), ("c128", False)):
        for _ in range(warmup):
            R.grad(args.qubits, c1, h1, p1[:1], complex64=c64, device='gpu')
        times = []
        for _ in range(count):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            R.grad(args.qubits, circ, ham, params[:1], complex64=c64, device='gpu')
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        out[prec] = times
    return out


def run_reference_gpu(args):
    """The reference's own thrust GPU simulator on this GPU: complex64 (the line's value) and
    complex128 (the reference's plain per-gate GPU path) full gradient evaluations."""
    from oracle import refbin as R

    if not R.available('gpu'):
        print(json.dumps({"impl": "reference", "unavailable": "the reference GPU simulator was not built "
                                                              "(make -C oracle refgpu, with the reference checkout)"}))
        return
    count = max(1, min(args.steps, 3))
    out = reference_gpu_evaluations(args, count, args.warmup)
    t = float(np.mean(out["c64"]))
    value = 1.0 / t
    sample = (f"full gradient evaluations (all {args.layers} layers, lambda = H psi) of parameter set 0, "
              f"{args.qubits} qubits, {count} timed per precision after {args.warmup} one-layer warm-ups")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": count, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic",
        "config": {"workload": f"HEA {args.qubits}q x {args.layers} layers, {2 * args.qubits * args.layers} params, "
                               f"{2 * args.qubits - 1}-term H, per-sample grad",
                   "n_qubits": args.qubits, "layers": args.layers, "batch": 1, "parallelism": "gpu x1"},
        "impl": "reference", "ref_device": "gpu: the reference's thrust mqvector_gpu built for sm_100a",
        "sample": sample, "seconds": out,
        "c128": {"value": 1.0 / float(np.mean(out["c128"])), "unit": UNIT},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(args, rank):
    if rank != 0:
        return
    if args.ref_device == 'gpu':
        run_reference_gpu(args)
        return
    threads = args.threads or os.cpu_count() or 1
    # a bounded run: at most three full evaluations (each tens of seconds on the host), plus
    # warm-up evaluations of one layer
    from oracle import refbin as R

    if R.available():
        c1, h1, p1 = build_workload(args.qubits, 1, args.batch)
        for _ in range(args.warmup):
            R.grad(args.qubits, c1, h1, p1[:1], threads=threads, complex64=True)
    count = max(1, min(args.steps, 3))
    times, kind = reference_full_evaluations(args.qubits, args.layers, args.batch, threads, count)
    t = float(np.mean(times))
    value = 1.0 / t
    sample = (f"full gradient evaluations (all {args.layers} layers, lambda = H psi, {2 * args.qubits * args.layers} "
              f"gradients) of parameter set 0, "
              f"{args.qubits} qubits complex64, {threads} host threads; {count} timed (of {args.steps} requested, "
              f"bounded), {args.warmup} one-layer warm-ups")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": count,
        "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"HEA {args.qubits}q x {args.layers} layers, {2 * args.qubits * args.layers} params, "
                               f"{2 * args.qubits - 1}-term H, per-sample grad",
                   "n_qubits": args.qubits, "layers": args.layers, "batch": 1, "parallelism": "cpu"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
                         "seconds": times},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["reference_gpu"] = _reference_gpu_extra(args)
    print(json.dumps(line), flush=True)


def _reference_gpu_extra(args):
    """Beside the CPU figure: the reference's own thrust GPU simulator on this box's GPU, one timed
    evaluation per precision after a one-layer warm-up (a few seconds), or why it did not run."""
    from oracle import refbin as R

    try:
        import torch

        if not (R.available('gpu') and torch.cuda.is_available()):
            return {"unavailable": "no GPU or the reference GPU simulator was not built"}
        out = reference_gpu_evaluations(args, 1, 1)
        return {"what": "the reference's thrust mqvector_gpu built for sm_100a, one evaluation of parameter set 0 "
                        "at a time", "unit": UNIT,
                "c64": 1.0 / float(np.mean(out["c64"])), "c128": 1.0 / float(np.mean(out["c128"])), "seconds": out}
    except Exception as e:  # pylint: disable=broad-except
        return {"unavailable": f"{type(e).__name__}: {e}"}


def run_b200(args, rank, world, local_rank):
    import torch

    from mindquantum_b200 import _native as N
    from mindquantum_b200 import complex64, complex128
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200
    from mindquantum_b200.simulator import lowering

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        import datetime

        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    dev = torch.device('cuda', local_rank)
    n, layers, B = args.qubits, args.layers, args.batch
    circ, ham, params_np = build_workload(n, layers, B, seed=rank)
    names = circ.params_name
    sim = MQVectorB200('mqvector_b200', n, dtype=complex64, device=dev)
    params = torch.as_tensor(params_np, device=dev)
    prog = lowering.lowered(circ, n, sim.precision, names, None, True)
    stride = sim._choose_stride(prog, B, 1)  # pylint: disable=protected-access
    n_passes, tile_bits = prog.grad_passes(1)

    def step():
        return sim.expectation_with_grad_tensor([ham], circ, params, names, ckpt_stride=stride)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            f, g = step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    value = world * B * args.steps / (ms / 1e3)

    # per-kernel event timing of the same steps (a separate timed run, so events do not perturb `value`)
    with N.KernelTimer() as kt:
        for _ in range(args.steps):
            step()
    launches = sum(kt.launches.values())
    dom = max(kt.ms, key=lambda k: kt.ms[k])
    S = (1 << n) * 8 * B
    n_ham = kt.launches['hamiltonian'] // args.steps
    # algorithmic bytes per step for each kernel kind
    alg = {
        'fused_forward': (2 * n_passes - 1) * S,                                 # pass 0 writes |0> tiles only
        'fused_backward': n_passes * 3 * S + (0 if stride == 1 else n_passes * S),  # psi read, lambda read+write
        'hamiltonian': (2 * S + 3 * S * (n_ham - 1)) if n_ham else 0,
    }
    peak, peak_kind = _peaks()
    achieved = alg.get(dom, 0) * args.steps / (kt.ms[dom] / 1e3) / 1e9 if kt.ms[dom] else None
    total_alg = sum(alg.values()) * args.steps
    traffic = ADJ_DRAM_BYTES_PER_STATE_BYTE
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (traffic * S if (traffic and dom == 'fused_backward') else None),
                "traffic_source": "ncu dram bytes per state byte of the adjoint pass (24-qubit capture) x S*B",
                "alg_bytes_per_launch": alg.get(dom, 0) / max(1, kt.launches[dom] // args.steps),
                "avg_launch_ms": kt.ms[dom] / max(1, kt.launches[dom]), "peak_source": peak_kind,
                "step_hbm_gbs": total_alg / (ms / 1e3) / 1e9 if world == 1 else None,
                "kernel_ms_per_step": {k: v / args.steps for k, v in kt.ms.items() if v}}

    # end to end through the public API: numpy in, numpy out (host<->device copies inside)
    ops = sim.get_expectation_with_grad(ham, circ)
    ops(params_np)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fe, ge = ops(params_np)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * B * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(params_np.nbytes),
           "d2h_bytes_per_step": int(fe.nbytes + ge.nbytes)}

    extras = {}
    if rank == 0 and not args.skip_extras:
        # accuracy: the same parameter set in complex128 (fused, FP64 throughout)
        s128 = MQVectorB200('mqvector_b200', n, dtype=complex128, device=dev)
        p1 = params[:1]
        s128.expectation_with_grad_tensor([ham], circ, p1, names, ckpt_stride=0)   # compiles the pass kernels
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f128, g128 = s128.expectation_with_grad_tensor([ham], circ, p1, names, ckpt_stride=0)
        torch.cuda.synchronize()
        t128 = time.perf_counter() - t0
        extras["grad_err_vs_c128"] = float((g[:1] - g128).abs().max().item())
        extras["f_err_vs_c128"] = float((f[:1, :, 0] - f128[:, :, 0]).abs().max().item())
        extras["grad_max_abs"] = float(g128.abs().max().item())
        extras["c128_fused"] = {"value": 1.0 / t128, "unit": UNIT, "batch": 1}
        extras.update(oracle_fixture_errors(n, layers, B, rank, f[0, 0, 0].item(), g[0, 0].cpu().numpy(),
                                            f128[0, 0, 0].item(), g128[0, 0].cpu().numpy()))
        checks = sim.norm_checks()   # the last timed step's FP64 norm checks (complex64 state)
        extras["norm_check"] = {"checks": int(checks.shape[0]), "states_per_check": B,
                                "max_abs_norm2_minus_1": float(np.max(np.abs(checks - 1.0))) if checks.size else None,
                                "cadence": "after every ceil(sqrt(passes))-th forward pass and the last"}
        extras["apply"] = apply_throughput(sim, circ, names, params, n, B, 5, peak)
        extras["device_error"] = N.device_error()
        if not args.skip_plain:
            # the plain complex128 single-circuit path: one kernel per gate, per-gate reductions
            sp = MQVectorB200('mqvector_b200', n, dtype=complex128, device=dev, fuse=False)
            sp.expectation_with_grad_tensor([ham], circ, p1, names, ckpt_stride=0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fp, gp = sp.expectation_with_grad_tensor([ham], circ, p1, names, ckpt_stride=0)
            torch.cuda.synchronize()
            tp = time.perf_counter() - t0
            extras["c128_plain"] = {"value": 1.0 / tp, "unit": UNIT, "batch": 1,
                                    "grad_err_vs_c128_fused": float((gp - g128).abs().max().item())}
            extras["ratio_vs_c128_plain"] = value / world / extras["c128_plain"]["value"]
            del sp
        del s128
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        times, kind = reference_full_evaluations(n, layers, B, threads, 1)
        cpu = {"value": 1.0 / times[0], "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"one full gradient evaluation (all {layers} layers, lambda = H psi) of parameter set 0, "
                         f"{n} qubits complex64: {times[0]:.1f} s"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": f"HEA {n}q x {layers} layers (RY,RZ + CNOT ladder), {len(names)} params, "
                                   f"51-term ZZ+X Hamiltonian, batched adjoint gradient",
                       "n_qubits": n, "layers": layers, "params": len(names), "batch_per_gpu": B,
                       "global_batch": B * world, "precision": "complex64 state, FP64 reductions",
                       "passes": n_passes, "tile_bits": tile_bits, "ckpt_stride": stride,
                       "l2": "inputs larger than L2 (512 MiB per state)", "parallelism": f"replicas x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
            "gpu_launches": launches, **extras,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_workload(args, rank, local_rank):
    """The other workload families on one GPU: the same JSON line, device-timed.

    qnn: 20-qubit RX-encoder QNN, 512 samples, Z_0..Z_3 (grad evals/s = samples/s with all four
    expectations and gradients); qaoa: MaxCut QAOA, 30 qubits, p = 10 on a 3-regular graph
    (complex64, error against complex128); uneven: 64 circuits of 12..24 qubits (U3 layers and
    brick CNOTs, own 10-term Hamiltonians) through one graph-captured CircuitBatch.
    """
    import torch

    from mindquantum_b200 import _native as N
    from mindquantum_b200 import complex64, complex128, workloads as W
    from mindquantum_b200.simulator.mqvector_b200 import MQVectorB200

    torch.cuda.set_device(local_rank)
    dev = torch.device('cuda', local_rank)
    extras = {}
    if args.workload == 'qnn':
        n, layers, B = 20, 6, 512
        circ, hams, enc, ans = W.qnn(n, layers, B, seed=rank)
        names = circ.params_name
        params_np = np.concatenate([enc, np.broadcast_to(ans, (B, len(ans)))], axis=1)
        params = torch.as_tensor(params_np, device=dev)
        sim = MQVectorB200('mqvector_b200', n, dtype=complex64, device=dev)
        units = B

        def step():
            return sim.expectation_with_grad_tensor(hams, circ, params, names)

        def e2e_step():
            return sim.get_expectation_with_grad(hams, circ)(enc, ans)

        io = (params_np.nbytes, B * len(hams) * (1 + len(names)) * 16)
        cfg = {"workload": f"QNN {n}q, RX encoder + {layers} x (RY, RZ, CZ ring), {len(names) - n} ansatz params, "
                           f"Z_0..Z_3, {B} samples", "n_qubits": n, "batch": B}
    elif args.workload == 'qaoa':
        n, p = 30, 10
        circ, ham, pr, edges = W.qaoa_maxcut(n, p, seed=rank)
        names = circ.params_name
        params = torch.as_tensor(pr[None, :], device=dev)
        sim = MQVectorB200('mqvector_b200', n, dtype=complex64, device=dev)
        units = 1

        def step():
            return sim.expectation_with_grad_tensor([ham], circ, params, names)

        def e2e_step():
            return sim.get_expectation_with_grad(ham, circ)(pr)

        io = (pr.nbytes, (1 + len(names)) * 16)
        cfg = {"workload": f"QAOA MaxCut {n}q, p={p}, 3-regular graph with {len(edges)} edges, H = sum Z_i Z_j",
               "n_qubits": n, "batch": 1}
    elif args.workload == 'csr':
        import scipy.sparse as sp  # noqa: F401
        from mindquantum_b200.core.operators import Hamiltonian
        from mindquantum_b200.simulator.lowering import native_ham

        n, layers, B = 22, 6, 8
        circ, ham_p, params_np = build_workload(n, layers, B, seed=rank)
        names = circ.params_name
        ham = Hamiltonian(W.pauli_csr(ham_p, n, np.complex64))
        params = torch.as_tensor(params_np, device=dev)
        sim = MQVectorB200('mqvector_b200', n, dtype=complex64, device=dev)
        units = B

        def step():
            return sim.expectation_with_grad_tensor([ham], circ, params, names)

        def e2e_step():
            return sim.get_expectation_with_grad(ham, circ)(params_np)

        io = (params_np.nbytes, B * (1 + len(names)) * 16)
        nnz = ham.sparse_matrix.nnz
        cfg = {"workload": f"HEA {n}q x {layers} layers, {len(names)} params, the ZZ+X Hamiltonian as a CSR matrix "
                           f"({nnz} entries), batched adjoint gradient", "n_qubits": n, "batch": B, "nnz": int(nnz)}
        # the CSR kernel alone: <psi_b|A|psi_b> of B resident states (matrix and states larger than L2)
        nh = native_ham(ham, n, sim.precision)
        states = torch.randn((B, 1 << n), dtype=torch.complex64, device=dev)
        out = torch.zeros((B, 2), dtype=torch.float64, device=dev)
        call = lambda: N.call('mqb_expectation', nh.handle, ctypes.c_void_p(states.data_ptr()),  # noqa: E731
                              ctypes.c_void_p(states.data_ptr()), B, ctypes.c_void_p(out.data_ptr()),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        for _ in range(3):
            call()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        c0.record()
        for _ in range(reps):
            call()
        c1.record()
        torch.cuda.synchronize()
        csr_ms = c0.elapsed_time(c1) / reps
        S = (1 << n) * 8
        passes = (B + 3) // 4
        alg = passes * (nnz * 12 + 8 * ((1 << n) + 1)) + B * 2 * S
        peak, peak_kind = _peaks()
        extras["csr_kernel"] = {"ms_per_call": csr_ms, "alg_bytes_per_call": int(alg),
                                "achieved_gbs": alg / (csr_ms / 1e3) / 1e9, "peak_gbs": peak, "peak_source": peak_kind,
                                "frac": alg / (csr_ms / 1e3) / 1e9 / peak, "states": B,
                                "bytes_model": "passes*(nnz*(4+8) + 8*(dim+1)) + B*2*S, passes = ceil(B/4)"}
        del states
    elif args.workload == 'noise':
        from mindquantum_b200.core import gates as G
        from mindquantum_b200.core.circuit import Circuit
        from mindquantum_b200.simulator import Simulator

        n, layers = 20, 4
        circ, ham, params_np = build_workload(n, layers, 1, seed=rank)
        noisy = Circuit()
        per_layer = 3 * n - 1
        for k, g in enumerate(circ):
            noisy += g
            if (k + 1) % per_layer == 0:     # after every layer: depolarizing + amplitude damping per qubit
                for q in range(n):
                    noisy += G.DepolarizingChannel(0.01).on(q)
                    noisy += G.AmplitudeDampingChannel(0.02).on(q)
        for q in range(n):
            noisy += G.Measure(f'q{q}').on(q)
        names = circ.params_name
        prd = dict(zip(names, params_np[0].tolist()))
        sim_api = Simulator('mqvector_b200', n, dtype=complex64, seed=7)
        shots = 1024
        units = shots
        seeds = iter(range(1, 1 << 30))

        def step():
            return sim_api.sampling(noisy, pr=prd, shots=shots, seed=next(seeds))

        e2e_step = step
        io = (params_np.nbytes, shots * n * 8)
        cfg = {"workload": f"noisy sampling, HEA {n}q x {layers} layers with a depolarizing (p=0.01) and an "
                           f"amplitude-damping (gamma=0.02) channel on every qubit after every layer "
                           f"({2 * n * layers} channels) and {n} measurements; {shots} shots per step, every "
                           f"shot one trajectory on its own stream, run as one batch", "n_qubits": n,
               "batch": shots}
    elif args.workload == 'pshift':
        n, layers = 16, 2
        circ, ham, params_np = build_workload(n, layers, 1, seed=rank)
        names = circ.params_name
        sim_api = None
        from mindquantum_b200.simulator import Simulator

        sim_api = Simulator('mqvector_b200', n, dtype=complex64)
        ops = sim_api.get_expectation_with_grad(ham, circ, pr_shift=True)
        units = 1

        def step():
            return ops(params_np[0])

        e2e_step = step
        io = (params_np.nbytes, (1 + len(names)) * 16)
        cfg = {"workload": f"parameter-shift gradient, HEA {n}q x {layers} layers, {len(names)} params "
                           f"({2 * len(names) + 1} shifted circuits as one batch)", "n_qubits": n, "batch": 1}
        adj = sim_api.get_expectation_with_grad(ham, circ)
        f_a, g_a = adj(params_np[0])
        f_s, g_s = ops(params_np[0])
        extras["grad_err_vs_adjoint"] = float(np.abs(g_s - g_a).max())
    else:
        from mindquantum_b200.simulator.batch import CircuitBatch

        members = W.uneven_u3(64, 12, 24, 20, seed=rank)
        batch = CircuitBatch([(m, c, h) for m, c, h, _ in members], dtype=complex64)
        plist = [torch.as_tensor(x, device=dev) for _, _, _, x in members]
        units = len(members)

        def step():
            return batch(plist)

        host_params = [x for _, _, _, x in members]

        def e2e_step():
            return batch.evaluate(host_params)

        io = (sum(x.nbytes for _, _, _, x in members), sum(16 * (1 + len(c.params_name)) for _, c, _, _ in members))
        cfg = {"workload": "64 circuits of 12..24 qubits, 20 x (U3 on every qubit + brick CNOTs), own 10-term "
                           "random Pauli Hamiltonians, one CUDA graph per call, autotuned tile widths",
               "n_circuits": len(members), "qubits": [m for m, _, _, _ in members], "graph_launches_per_call": 1,
               "kernel_launches_per_call": batch.launches_per_call()}
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = units * args.steps / (ms / 1e3)
    with N.KernelTimer() as kt:
        for _ in range(args.steps):
            step()
    torch.cuda.synchronize()   # launches replayed from a graph are not timed: finish them first
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if args.workload == 'qaoa' and not args.skip_extras:
        f64, g64 = step()
        s128 = MQVectorB200('mqvector_b200', 30, dtype=complex128, device=dev)
        f128, g128 = s128.expectation_with_grad_tensor([ham], circ, params, names)
        extras["grad_err_vs_c128"] = float((g64 - g128).abs().max().item())
        extras["f_err_vs_c128"] = float((f64[..., 0] - f128[..., 0]).abs().max().item())
        del s128
    unit = "trajectories/s" if args.workload == 'noise' else UNIT
    # kernels inside a replayed graph are not seen by the per-launch timer: count the recorded ones
    launches = cfg.get("kernel_launches_per_call", 0) * args.steps or sum(kt.launches.values())
    line = {
        "metric": f"{unit}, {args.workload} workload", "value": value, "unit": unit, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic", "config": cfg,
        "e2e": {"value": units * args.steps / e2e_s, "unit": unit, "h2d_bytes_per_step": int(io[0]),
                "d2h_bytes_per_step": int(io[1])},
        "kernel_ms_per_step": {k: v / args.steps for k, v in kt.ms.items() if v},
        "clocks": clocks.summary(), "gpu_launches": launches, **extras,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--qubits', type=int, default=26)
    ap.add_argument('--layers', type=int, default=12)
    ap.add_argument('--batch', type=int, default=8)
    ap.add_argument('--skip-extras', action='store_true')
    ap.add_argument('--threads', type=int, default=0,
                    help='host threads of the reference arm (default: every core)')
    ap.add_argument('--ref-device', default='cpu', choices=['cpu', 'gpu'],
                    help="reference arm: the reference's CPU simulator (default) or its thrust GPU simulator")
    ap.add_argument('--skip-plain', action='store_true')
    ap.add_argument('--skip-cpu', action='store_true')
    ap.add_argument('--workload', default='hea', choices=['hea', 'qnn', 'qaoa', 'uneven', 'csr', 'pshift', 'noise'],
                    help='hea: the headline 26-qubit HEA gradient; the others are the remaining workload families')
    args = ap.parse_args()
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local_rank = int(os.environ.get('LOCAL_RANK', 0))
    if args.impl == 'reference':
        run_reference(args, rank)
        return
    if args.workload != 'hea':
        if rank == 0:
            run_workload(args, rank, local_rank)
        return
    run_b200(args, rank, world, local_rank)


if __name__ == '__main__':
    main()
