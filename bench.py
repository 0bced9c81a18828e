#!/usr/bin/env python
"""Throughput of the dynamical-core step and its gradient on B200:
cell-steps/s of forward + adjoint.

One step is one model step of run_model (src/mod_model.f90:146-177): the
C-grid half step, its halo fill, the D-grid step, the vertical remap when
due (every 8 steps) and the D-grid halo fill.  One cell-step is one
interior (i, j, k) cell advanced by one such step.

Workload: the seeded zonal-jet case at 1024 x 1024 x 64 (dx = 25 km,
dt = 30 s, remap every 8 steps), synthetic data from atmdyn.ic.jet_case.
The headline ``value`` is forward + adjoint of the FP64 form through the
torch.autograd binding: K steps forward with checkpoints every 8 steps,
J = sum(theta^2) over the final state (every tile of the adjoint active),
and the hand-written adjoint back to the initial state, per (K cells x
steps) / (forward + backward time).  Beside it: the FP64 and mixed forward
forms (``forms``), the masked loss of the differentiation case and its
finite-difference check (``adjoint``), the batched ensemble, the column
physics, the radiation, and CPU baselines of the reference algorithm (the FP64
restatement: forward plus its tangent-linear model, which stands in for a
reverse pass since the reference has no derivative code).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank advances its own replica of the domain
(the path shards, but one domain fits one GPU; replicas only) and the time
is the maximum over ranks.  ``--impl reference`` times the reference's CPU
algorithm (the FP64 restatement, forward + tangent-linear pass) on the
host cores, on a 256 x 256 x 64 sample of the same case.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'atmosphere-model_b200'))

import numpy as np  # noqa: E402

METRIC = 'cell-steps/s fwd+adjoint on 1 B200 vs FP64 form, % HBM roofline, err vs FP64'
NX = NY = 1024
NLAY = 64
DT = 30.0
REMAP_EVERY = 8
ADJ_CKPT = 8
SAMPLE_N = 256

# Algorithmic HBM words per interior cell and launch of each kernel: every
# field the kernel must read or write once (layer-nlay slabs and halo rings
# are excluded), split by storage type: (state words, C-grid words, fp64
# words).  The state (dp, pt, ud, vd) is FP64 in both forms; the C-grid
# fields (dpc, ptc, uc, vc) are FP64 in the FP64 form and FP32 in the mixed
# form; pkap, gz, pkapb, gzb are FP64.
WORDS = {
    'c_mass': (4, 2, 0),        # read dp, pt, ud, vd; write dpc, ptc
    'c_column': (0, 2, 2),      # read dpc, ptc; write pkap, gz
    'c_mom': (2, 2, 2),         # read ud, vd, pkap, gz; write uc, vc
    'd_mass': (4, 2, 0),        # read dp, pt, uc, vc; write dp, pt
    'd_column': (2, 0, 2),      # read dp, pt; write pkap, gz
    'd_corners': (0, 0, 4),     # read pkap, gz; write pkapb, gzb
    'd_mom': (4, 2, 2),         # read ud, vd, uc, vc, pkapb, gzb; write ud, vd
    'remap_winds': (5, 0, 0),   # read dp, ud, vd; write u, v remapped
    'remap_energy': (10, 0, 0),  # read dp, pt, ud, vd, u, v remapped; write dp, pt, ud, vd
    'phys_tend': (7, 0, 0),     # read dp, pt, ud, vd; write pt, u, v tendencies
    'phys_apply': (11, 0, 0),   # read dp, pt, ud, vd and the three tendencies; write dp, pt, ud, vd
}


def kernel_bytes(stage, form, cells):
    w_s, w_c, w_d = WORDS.get(stage, (0, 0, 0))
    ec = 8 if form == 'fp64' else 4
    return (w_s * 8 + w_c * ec + w_d * 8) * cells


# DRAM bytes per interior cell and launch measured by ncu on the FP64 form
# (dram__bytes_read.sum + dram__bytes_write.sum, jet 512x512x32, scaled by
# cells)
TRAFFIC_PER_CELL_FP64 = {'c_mass': 48.3, 'c_mom': 48.3, 'd_mass': 48.4, 'd_mom': 66.2, 'c_column': 31.4,
                         'd_column': 31.4}


def load_peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self):
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        try:
            self.p = subprocess.Popen(['nvidia-smi', '--query-gpu=' + self.Q, '--format=csv,noheader,nounits',
                                       '-lms', '200'], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(smax), 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_setup():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return world, rank, local


class Ranks:
    """Rank coordination of a run: a barrier, and the maximum of a device
    time over the ranks (every rank takes the same collective steps in the
    same order).  One rank: no collective."""

    def __init__(self, world, device):
        self.world, self.device = world, device

    def barrier(self):
        import torch
        if self.world > 1:
            torch.distributed.barrier()
        if self.device.type == 'cuda':
            torch.cuda.synchronize()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())


def cpu_grad_throughput(n, steps, warmup, threads):
    """The FP64 restatement of the reference on the host cores, on the jet
    case at n x n x NLAY (remap every REMAP_EVERY steps, counted from the
    first warm-up step): ``steps`` steps of the forward and ``steps`` steps
    of its tangent-linear model (dual numbers: the forward values and one
    directional derivative), after ``warmup`` untimed steps of each.  The
    reference has no derivative code; one tangent-linear pass stands in for
    the reverse pass of the GPU's forward + adjoint.  Returns the forward +
    derivative rate and the forward-only rate, cell-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import pyoracle
    from atmdyn import ic
    st = ic.jet_case(n, n, NLAY, 25e3, 25e3, seed=0)
    rng = np.random.default_rng(0)
    o = pyoracle.OracleModel(st, threads=threads)
    tl = pyoracle.TLMModel(st, {'pt': rng.normal(0, 1e-3, st.pt.shape)}, threads=threads)

    def run(m, first, count):
        for q in range(first, first + count):
            m.cgrid_step(DT / 2.)
            m.cgrid_halo()
            m.dgrid_step(DT)
            if (q + 1) % REMAP_EVERY == 0:
                m.remap()
            m.dgrid_halo()
        assert m.check_stability()

    run(o, 0, warmup)
    run(tl, 0, warmup)
    t0 = time.perf_counter()
    run(o, warmup, steps)
    tf = time.perf_counter() - t0
    t0 = time.perf_counter()
    run(tl, warmup, steps)
    tt = time.perf_counter() - t0
    remaps = sum(1 for q in range(warmup, warmup + steps) if (q + 1) % REMAP_EVERY == 0)
    return {'value': st.cells * steps / (tf + tt), 'forward_only': st.cells * steps / tf,
            'forward_s': tf, 'tangent_linear_s': tt, 'remaps': remaps}


def cpu_baseline_lines(steps, warmup):
    """All host cores on the 256^2 sample (the reference arm's workload) and
    one core on a 128^2 sample (8 steps with one remap)."""
    threads = len(os.sched_getaffinity(0))
    a = cpu_grad_throughput(SAMPLE_N, steps, warmup, threads)
    one = cpu_grad_throughput(SAMPLE_N // 2, REMAP_EVERY, 1, 1)
    out = {'value': a['value'], 'unit': 'cell-steps/s', 'cores': threads, 'kind': 'port',
           'sample': 'jet %dx%dx%d, %d steps forward + %d steps tangent-linear (%d remaps) after %d warm-up each' % (
               SAMPLE_N, SAMPLE_N, NLAY, steps, steps, a['remaps'], warmup),
           'forward_only': a['forward_only'],
           'single_core': {'value': one['value'], 'unit': 'cell-steps/s', 'cores': 1, 'kind': 'port',
                           'forward_only': one['forward_only'],
                           'sample': 'jet %dx%dx%d, %d steps forward + %d tangent-linear (%d remap) after 1 '
                                     'warm-up each' % (SAMPLE_N // 2, SAMPLE_N // 2, NLAY, REMAP_EVERY,
                                                       REMAP_EVERY, one['remaps'])}}
    return out


def headline_config(nx, nlay, steps, world):
    """The workload of the headline, the same in both arms' lines."""
    return {'workload': 'jet %dx%dx%d, dx=25 km, dt=30 s, remap every %d steps, FP64 form: %d steps forward '
                        '(checkpoints every %d) + adjoint of J = sum(theta^2) at the final step' % (
                            nx, nx, nlay, REMAP_EVERY, steps, ADJ_CKPT),
            'nx': nx, 'ny': nx, 'nlay': nlay, 'remap_every': REMAP_EVERY, 'checkpoint_every': ADJ_CKPT,
            'l2': 'inputs larger than L2 (each prognostic field is 552 MB)',
            'parallelism': 'replicas' if world > 1 else 'single GPU'}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    threads = len(os.sched_getaffinity(0))
    steps, warmup = args.steps, args.warmup
    r = cpu_grad_throughput(SAMPLE_N, steps, warmup, threads)
    v = r['value']
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'cell-steps/s', 'n_gpus': args.gpus,
        'steps': steps, 'warmup': warmup, 'ms_per_step': 1000 * (r['forward_s'] + r['tangent_linear_s']) / steps,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic (seeded jet case)',
        'config': headline_config(args.nx, args.nlay, steps, world),
        'cpu_baseline': {'value': v, 'unit': 'cell-steps/s', 'cores': threads, 'kind': 'port',
                         'sample': 'jet %dx%dx%d, %d steps forward + %d steps tangent-linear (%d remaps) after %d '
                                   'warm-up each (1/16 of the 1024^2 domain)' % (
                                       SAMPLE_N, SAMPLE_N, NLAY, steps, steps, r['remaps'], warmup),
                         'forward_only': r['forward_only']},
        'e2e': {'value': v, 'unit': 'cell-steps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=timedelta(seconds=300), device_id=torch.device('cuda', local))
    else:
        torch.cuda.set_device(0)
    from atmdyn import ic, Dycore
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    cells = st.cells
    K, W = args.steps, args.warmup
    peak, peak_kind = load_peaks()

    ranks = Ranks(world, torch.device('cuda', torch.cuda.current_device()))
    barrier, max_over_ranks = ranks.barrier, ranks.max

    results = {}
    states = {}
    clocks = None
    forms = args.forms.split(',')
    for form in forms:
        dy = Dycore(st, form)
        stream = torch.cuda.Stream()
        dy.set_stream(stream.cuda_stream)
        n = 0

        def one():
            nonlocal n
            n += 1
            return dy.step(DT, remap=(n % REMAP_EVERY == 0), check_stable=True)

        # every kernel of the step, the remap's included, launches once before
        # the warm-up (first-launch costs such as module loading stay out of
        # the timed region whatever W is): one step with remap from a saved
        # copy of the state, which is then restored
        saved = torch.empty(dy.state_bytes() // 8, dtype=torch.float64, device='cuda')
        dy.state_save(saved.data_ptr())
        dy.step(DT, remap=True, check_stable=False)
        dy.state_load(saved.data_ptr())
        dy.sync()
        del saved
        for _ in range(W):
            one()
        barrier()
        if form == 'fp64':
            clk = Clocks()
        l0 = dy.launch_count()
        dy.profile(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        stable = True
        for _ in range(K):
            stable = one() and stable
        e1.record(stream)
        torch.cuda.synchronize()
        if form == 'fp64':
            clocks = clk.stop()
        ms = max_over_ranks(e0.elapsed_time(e1))
        prof = dy.profile_read()
        dy.profile(False)
        launches = dy.launch_count() - l0
        barrier()
        kern = {}
        for stage, (tms, cnt) in prof.items():
            if cnt == 0:
                continue
            b = kernel_bytes(stage, form, cells)
            avg = tms / cnt
            kern[stage] = {'ms_avg': round(avg, 4), 'launches': cnt, 'share': round(tms / max(ms, 1e-9), 4)}
            if b:
                kern[stage]['algorithmic_bytes'] = b
                kern[stage]['gbs'] = round(b / (avg * 1e-3) / 1e9, 1)
        value = world * cells * K / (ms * 1e-3)
        results[form] = {'value': value, 'ms_per_step': ms / K, 'stable': stable, 'kernels': kern,
                         'gpu_launches': launches, 'steps_done': n}
        states[form] = dy.state()
        if form == 'fp64' and not args.no_e2e:
            results[form]['e2e'], results[form]['e2e_resident'] = e2e_runs(dy, st, K, stream, torch, max_over_ranks,
                                                                            world)
        dy.close()
        del dy
        torch.cuda.empty_cache()

    grad = grad_leg(args, torch, barrier, max_over_ranks, world, peak, peak_kind)
    adjoint = None if args.no_adjoint else adjoint_leg(args, torch, max_over_ranks, world)
    ensemble = None if (args.no_ensemble or world > 1) else ensemble_leg(args, torch)
    physics = None if args.no_physics else physics_leg(args, torch, max_over_ranks, world, peak, peak_kind)
    radiation = None if args.no_radiation else radiation_leg(args, torch, max_over_ranks, world)

    # error of the mixed form against the FP64 form after the same steps
    err = {}
    for name in (('dp', 'pt', 'ud', 'vd') if len(states) == 2 else ()):
        a, b = states['fp64'][name], states['mixed'][name]
        err[name] = {'rel_l2': float(np.linalg.norm(b - a) / max(np.linalg.norm(a), 1e-300)),
                     'rel_max': float(np.abs(b - a).max() / max(np.abs(a).max(), 1e-300))}

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    f64 = results['fp64'] if 'fp64' in results else next(iter(results.values()))
    mixed = results.get('mixed') if 'fp64' in results else None
    # the forward's dominant kernel, for the forward forms' own roofline
    fdom_name, fdom_k = max(f64['kernels'].items(), key=lambda kv: kv[1]['ms_avg'] * kv[1]['launches'])
    fwd_roofline = {'bound': 'hbm', 'kernel': fdom_name, 'achieved': fdom_k.get('gbs', 0.0), 'peak': peak,
                    'unit': 'GB/s', 'frac': fdom_k.get('gbs', 0.0) / peak, 'peak_kind': peak_kind,
                    'traffic': (TRAFFIC_PER_CELL_FP64[fdom_name] * cells if fdom_name in TRAFFIC_PER_CELL_FP64
                                else None)}
    line = {
        'metric': METRIC, 'value': grad['value'], 'unit': 'cell-steps/s', 'n_gpus': world, 'steps': K, 'warmup': W,
        'ms_per_step': grad['ms_per_step'], 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f64', 'data': 'synthetic (seeded jet case, atmdyn.ic.jet_case)',
        'config': headline_config(args.nx, args.nlay, K, world),
        'roofline': grad['roofline'],
        'e2e': grad['e2e'],
        'gpu_launches': grad['gpu_launches'],
        'clocks': grad['clocks'],
        'kernels': grad['kernels'],
        'forward_ms': grad['forward_ms'], 'backward_ms': grad['backward_ms'],
        'backward_over_forward': grad['backward_ms'] / grad['forward_ms'],
        'forms': {
            'fp64': {'value': f64['value'], 'unit': 'cell-steps/s (forward)', 'ms_per_step': f64['ms_per_step'],
                     'stable': f64['stable'], 'roofline': fwd_roofline, 'kernels': f64['kernels'],
                     'e2e': f64.get('e2e'), 'e2e_resident': f64.get('e2e_resident'),
                     'gpu_launches': f64['gpu_launches'], 'clocks': clocks},
        },
    }
    if mixed:
        line['forms']['mixed'] = {'value': mixed['value'], 'unit': 'cell-steps/s (forward)',
                                  'ms_per_step': mixed['ms_per_step'],
                                  'stable': mixed['stable'], 'speedup_vs_fp64': mixed['value'] / f64['value'],
                                  'err_vs_fp64_after_%d_steps' % (K + W): err, 'kernels': mixed['kernels']}
    if adjoint is not None:
        line['adjoint'] = adjoint
    if ensemble is not None:
        line['ensemble'] = ensemble
    if physics is not None:
        line['physics'] = physics
    if radiation is not None:
        line['radiation'] = radiation
    if world == 1 and not args.no_cpu:
        line['cpu_baseline'] = cpu_baseline_lines(K, W)
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


P0K = 1.0e5 ** (287.052874 / 1005.0)  # theta = pt * p0**kappa


def physics_leg(args, torch, max_over_ranks, world, peak, peak_kind):
    """The column physics (src/mod_physics.f90, FP64) on the headline
    workload: calculate_physics_tendencies (k_physics_tend) and
    apply_physics_tendencies (k_physics_apply), each launch timed with CUDA
    events on the context's stream, and the FP64 restatement of the same two
    routines on one host core on a 256 x 256 x 64 sample."""
    from atmdyn import ic, Dycore
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    st.ts = np.full((st.ny, st.nx), 288.0)
    cells = st.cells
    dy = Dycore(st)
    stream = torch.cuda.Stream()
    dy.set_stream(stream.cuda_stream)
    for _ in range(3):
        dy.physics_tendencies()
        dy.apply_physics(DT)
        dy.physics_halo()
    torch.cuda.synchronize()
    reps = 8
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dy.profile(True)
    e0.record(stream)
    for _ in range(reps):
        dy.physics_tendencies()
        dy.apply_physics(DT)
        dy.physics_halo()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1)) / reps
    prof = dy.profile_read()
    dy.profile(False)
    dy.close()
    del dy
    torch.cuda.empty_cache()
    kern = {}
    for stage, (tms, cnt) in prof.items():
        if cnt == 0:
            continue
        avg = tms / cnt
        kern[stage] = {'ms_avg': round(avg, 4), 'launches': cnt}
        b = kernel_bytes(stage, 'fp64', cells)
        if b:
            kern[stage].update({'algorithmic_bytes': b, 'gbs': round(b / (avg * 1e-3) / 1e9, 1),
                                'frac_of_peak': round(b / (avg * 1e-3) / 1e9 / peak, 3)})
    out = {'workload': 'jet %dx%dx%d, tendencies + application + ts halo per call' % (args.nx, args.nx, args.nlay),
           'ms_per_call': ms, 'cells_per_s': world * cells / (ms * 1e-3), 'kernels': kern,
           'peak_gbs': peak, 'peak_kind': peak_kind}
    if world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, 'oracle'))
        import pyoracle
        sm = ic.jet_case(SAMPLE_N, SAMPLE_N, args.nlay, 25e3, 25e3, seed=0)
        sm.ts = np.full((sm.ny, sm.nx), 288.0)
        o = pyoracle.OracleModel(sm)
        o.physics_tendencies()
        o.apply_physics(DT)
        t0 = time.perf_counter()
        n = 2
        for _ in range(n):
            o.physics_tendencies()
            o.apply_physics(DT)
            o.physics_halo()
        t = time.perf_counter() - t0
        out['cpu_baseline'] = {'value': sm.cells * n / t, 'unit': 'cells/s', 'cores': 1, 'kind': 'port',
                               'sample': 'jet %dx%dx%d, %d calls after 1 warm-up' % (SAMPLE_N, SAMPLE_N,
                                                                                     args.nlay, n)}
    return out


def radiation_leg(args, torch, max_over_ranks, world):
    """The radiation (src/mod_radiation.f90, FP64) on the headline workload:
    calculate_radiative_heating (k_radiation: per column the layer
    temperatures, then 16 g-points of shortwave and longwave two-stream
    solutions closed by the adding method) and the net-flux halo, timed with
    CUDA events on the context's stream; the reference's tables when the
    package build extracted them, else synthetic ones of the same shapes.
    The FP64 restatement of the same routine runs on a 64 x 64 sample of
    columns on one host core and on all of them."""
    from atmdyn import ic, Dycore, gas_optics
    go = gas_optics.load_default()
    tables = 'reference (extracted)' if go is not None else 'synthetic'
    go = go or gas_optics.synthetic(0)
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    st.ts = np.full((st.ny, st.nx), 288.0)
    cols = st.nx * st.ny
    dy = Dycore(st)
    dy.set_radiation(go)
    stream = torch.cuda.Stream()
    dy.set_stream(stream.cuda_stream)
    dy.radiative_heating()
    torch.cuda.synchronize()
    reps = 3
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    dy.profile(True)
    e0.record(stream)
    for _ in range(reps):
        dy.radiative_heating()
        dy.radiation_halo()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1)) / reps
    prof = dy.profile_read()
    dy.profile(False)
    dy.close()
    del dy
    torch.cuda.empty_cache()
    kern = {k: {'ms_avg': round(t / c, 4), 'launches': c} for k, (t, c) in prof.items() if c}
    ng = go.n_g
    out = {'workload': 'jet %dx%dx%d, %d g-points, tables: %s; one call + net-flux halo' % (
               args.nx, args.nx, args.nlay, ng, tables),
           'ms_per_call': ms, 'columns_per_s': world * cols / (ms * 1e-3),
           'layer_gpoints_per_s': world * cols * args.nlay * ng / (ms * 1e-3), 'kernels': kern}
    if world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, 'oracle'))
        import pyoracle
        n = 64
        sm = ic.jet_case(n, n, args.nlay, 25e3, 25e3, seed=0)
        ts = np.full((n, n), 288.0)
        xc, yc = ic.cell_axes(sm)
        threads = len(os.sched_getaffinity(0))
        base = {}
        for cores in sorted({1, threads}):
            t0 = time.perf_counter()
            pyoracle.radiative_heating(go, sm.dp, sm.pt, ts, xc, yc, sm.ak[0], sm.gravity, threads=cores)
            base[cores] = n * n / (time.perf_counter() - t0)
        out['cpu_baseline'] = [{'value': v, 'unit': 'columns/s', 'cores': c, 'kind': 'port',
                                'sample': 'jet %dx%dx%d, one call' % (n, n, args.nlay)} for c, v in base.items()]
    return out


def probe_radiation(args):
    """A small case for ncu captures of the radiation kernel (nothing is
    timed here): a jet at nx x nx x nlay, three calls."""
    import torch
    torch.cuda.set_device(0)
    from atmdyn import ic, Dycore, gas_optics
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    st.ts = np.full((st.ny, st.nx), 288.0)
    dy = Dycore(st)
    dy.set_radiation(gas_optics.load_default() or gas_optics.synthetic(0))
    for _ in range(3):
        dy.radiative_heating()
    dy.close()
    print('radiation probe done: %dx%dx%d' % (args.nx, args.nx, args.nlay))


# Algorithmic HBM words per interior cell and launch of the adjoint
# kernels: the forward inputs the kernel recomputes from, the output
# adjoints it reads, and a read and a write of every adjoint it adds into
# (layer-nlay slabs excluded, as for the forward).
ADJ_WORDS = {
    'adj_c_mass': 14,    # dp, pt, ud, vd; lam dpc, ptc; += lam dp, pt, ud, vd
    'adj_c_mom': 14,     # ud, vd, pkap, gz; lam uc, vc; += lam ud, vd, pkap, gz
    'adj_d_mom_ke': 8,   # ud, vd; lam ud, vd (out); += lam ud, vd (in)
    'adj_d_mom_vf': 20,  # ud, vd, uc, vc, pkapb, gzb; lam ud, vd (out); += lam ud, vd, uc, vc, pkapb, gzb
    'adj_d_mass_x': 16,  # dp, pt, uc, vc, new dp, pt; lam dp, pt (out); += lam dp, pt, uc, vc
    'adj_d_mass_y': 16,
}
# DRAM bytes per interior cell and launch of the adjoint kernels measured by
# ncu (dram__bytes_read.sum + dram__bytes_write.sum, dense adjoint of the
# jet at 512x512x32, scaled by cells)
TRAFFIC_PER_CELL_ADJ = {'adj_c_mass': 113.3, 'adj_c_mom': 114.2, 'adj_d_mass_x': 130.9, 'adj_d_mass_y': 131.1,
                        'adj_d_mom_ke': 64.7, 'adj_d_mom_vf': 165.2}


def grad_leg(args, torch, barrier, max_over_ranks, world, peak, peak_kind):
    """The headline: the gradient of J = sum(theta^2) over the final state
    (theta = pt p0**kappa) with respect to the initial dp, pt, ud, vd,
    through atmdyn.adjoint.integrate (FP64 form, checkpoints every ADJ_CKPT
    steps, the last segment's tapes recorded by its forward).  W steps of
    forward + adjoint untimed, then exactly K steps timed (forward and
    backward separately, CUDA events on torch's current stream, which the
    library is bound to); one more identical pass with per-launch events for
    the per-kernel breakdown and the roofline of the dominant kernel; one
    pass end to end from and to pinned host memory."""
    from atmdyn import ic, Dycore
    from atmdyn.adjoint import integrate
    K, W = args.steps, args.warmup
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    st.dt = DT
    cells = st.cells
    dyn = Dycore(st)
    dyn.adj_enable()
    inputs = [torch.tensor(np.ascontiguousarray(a), device='cuda') for a in (st.dp, st.pt, st.u, st.v)]

    def fwd_bwd(nsteps, x, events=None):
        if events:
            events[0].record()
        y = integrate(dyn, x, nsteps, DT, REMAP_EVERY, ADJ_CKPT)
        J = ((y[1] * P0K) ** 2).sum()
        if events:
            events[1].record()
        J.backward()
        if events:
            events[2].record()
        return J

    def fresh():
        return [t.clone().requires_grad_(True) for t in inputs]

    fwd_bwd(W, fresh())  # warm-up: W steps forward + adjoint
    torch.cuda.synchronize()
    x = fresh()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    barrier()
    l0 = dyn.launch_count()
    clk = Clocks()
    J = fwd_bwd(K, x, ev)
    barrier()
    clocks = clk.stop()
    launches = dyn.launch_count() - l0
    tf = max_over_ranks(ev[0].elapsed_time(ev[1]))
    tb = max_over_ranks(ev[1].elapsed_time(ev[2]))
    gnorm = float(sum(float(xx.grad.norm()) ** 2 for xx in x) ** .5)
    # the same pass with per-launch events (stage breakdown, roofline)
    del x
    x = fresh()
    torch.cuda.synchronize()
    dyn.profile(True)
    fwd_bwd(K, x)
    torch.cuda.synchronize()
    prof = dyn.profile_read()
    dyn.profile(False)
    del x
    kern = {}
    for stage, (tms, cnt) in prof.items():
        if cnt == 0:
            continue
        avg = tms / cnt
        kern[stage] = {'ms_avg': round(avg, 4), 'launches': cnt, 'share': round(tms / max(tf + tb, 1e-9), 4)}
        words = ADJ_WORDS.get(stage)
        b = words * 8 * cells if words else kernel_bytes(stage, 'fp64', cells)
        if b:
            kern[stage]['algorithmic_bytes'] = b
            kern[stage]['gbs'] = round(b / (avg * 1e-3) / 1e9, 1)
    # dominant kernel: the single-kernel stage with the largest total time
    single = {k: v for k, v in kern.items() if k in ADJ_WORDS or k in WORDS}
    dom_name, dom = max(single.items(), key=lambda kv: kv[1]['ms_avg'] * kv[1]['launches'])
    achieved = dom.get('gbs', 0.0)
    roofline = {'bound': 'hbm', 'kernel': dom_name, 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                'frac': achieved / peak, 'peak_kind': peak_kind,
                'traffic': (TRAFFIC_PER_CELL_ADJ[dom_name] * cells if dom_name in TRAFFIC_PER_CELL_ADJ else
                            TRAFFIC_PER_CELL_FP64[dom_name] * cells if dom_name in TRAFFIC_PER_CELL_FP64 else None),
                'traffic_unit': 'bytes per launch (ncu DRAM read + write per cell, scaled by cells)',
                'algorithmic_bytes_per_launch': dom.get('algorithmic_bytes'),
                'ms_per_launch': dom['ms_avg'], 'launches': dom['launches']}
    # end to end: the inputs from pinned host memory, the loss and the four
    # gradients back to pinned host memory, inside the timed region
    host_in = [torch.empty(t.shape, dtype=torch.float64, pin_memory=True) for t in inputs]
    host_out = [torch.empty(t.shape, dtype=torch.float64, pin_memory=True) for t in inputs]
    for h, t in zip(host_in, inputs):
        h.copy_(t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record()
    x = [torch.empty_like(t).copy_(h, non_blocking=True).requires_grad_(True) for t, h in zip(inputs, host_in)]
    J2 = fwd_bwd(K, x)
    for h, xx in zip(host_out, x):
        h.copy_(xx.grad, non_blocking=True)
    j_host = J2.item()
    e1.record()
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1))
    nbytes = sum(h.numel() * 8 for h in host_in)
    e2e = {'value': world * cells * K / (ms_e2e * 1e-3), 'unit': 'cell-steps/s', 'h2d_bytes_per_step': nbytes / K,
           'd2h_bytes_per_step': (nbytes + 8) / K, 'steps': K,
           'how': 'one pass of K steps: dp, pt, ud, vd copied from pinned host memory, forward + adjoint through '
                  'atmdyn.adjoint.integrate, J and the four gradients copied back to pinned host memory',
           'same_gradient_as_device_timed': bool(abs(j_host - J.item()) <= 1e-12 * abs(J.item()))}
    dyn.close()
    del dyn, x, J, J2
    torch.cuda.empty_cache()
    return {'value': world * cells * K / ((tf + tb) * 1e-3), 'ms_per_step': (tf + tb) / K, 'forward_ms': tf,
            'backward_ms': tb, 'gpu_launches': launches, 'clocks': clocks, 'kernels': kern, 'roofline': roofline,
            'e2e': e2e, 'grad_norm': gnorm}


def adjoint_leg(args, torch, max_over_ranks, world):
    """fwd+adjoint through atmdyn.adjoint.integrate with the masked loss of
    the differentiation case on the headline workload, and the timing and
    finite-difference check of the differentiation case itself: 512 x 512 x 32
    jet (seed 2), 20 steps, checkpoints every 5, J = sum(mask theta^2) at
    the final step with a 300 km Gaussian mask at mid-domain, central
    differences with eps = 1e-6 along 8 seeded random unit directions."""
    from atmdyn import ic, Dycore
    from atmdyn.adjoint import integrate, gaussian_mask
    out = {}

    def timed(st, nsteps, remap_every, ckpt, reps, dense=False):
        dyn = Dycore(st)
        dyn.adj_enable()
        mask = gaussian_mask(st, 300e3, device='cuda')
        if dense:  # J = sum(theta^2): the adjoint is non-zero everywhere from the first reverse step
            mask = torch.ones_like(mask)
        x = [torch.tensor(np.ascontiguousarray(a), device='cuda', requires_grad=True)
             for a in (st.dp, st.pt, st.u, st.v)]

        def final_theta(fields):
            return integrate(dyn, fields, nsteps, st.dt, remap_every, ckpt)[1] * P0K

        def loss(fields):
            return (mask * final_theta(fields) ** 2).sum()

        J = loss(x)  # warm-up (tensor maps, allocator)
        J.backward()
        best = None
        # timed passes without the per-launch profiling events, then one
        # profiled pass for the per-stage breakdown
        for rep in range(reps + 1 if reps else 0):
            profiled = rep == reps
            for xx in x:
                xx.grad = None
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            dyn.profile(profiled)
            l0 = dyn.launch_count()
            clk = Clocks()
            ev[0].record()
            J = loss(x)
            ev[1].record()
            J.backward()
            ev[2].record()
            torch.cuda.synchronize()
            clocks = clk.stop()
            tf = max_over_ranks(ev[0].elapsed_time(ev[1]))
            tb = max_over_ranks(ev[1].elapsed_time(ev[2]))
            if profiled:
                prof = {k: (round(v[0], 3), v[1]) for k, v in dyn.profile_read().items() if v[1]}
                dyn.profile(False)
                best = best[:2] + (prof,) + best[3:]
            elif best is None or tf + tb < best[0] + best[1]:
                best = (tf, tb, None, dyn.launch_count() - l0, clocks)
        return dyn, x, final_theta, mask, J, best

    # the headline workload with the masked loss of the differentiation case
    # (a loss over a sub-domain: tiles outside its domain of dependence skip)
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    st.dt = DT
    nsteps = args.steps
    try:
        dyn, x, _, _, J, (tf, tb, prof, launches, clocks) = timed(st, nsteps, REMAP_EVERY, ADJ_CKPT, 1)
        cells = st.cells
        out['masked_loss'] = {
            'value': world * cells * nsteps / ((tf + tb) * 1e-3), 'unit': 'cell-steps/s (forward + adjoint)',
            'workload': 'jet %dx%dx%d, %d steps, remap every %d, checkpoints every %d, J = sum(mask theta^2), '
                        '300 km Gaussian mask' % (args.nx, args.nx, args.nlay, nsteps, REMAP_EVERY, ADJ_CKPT),
            'forward_ms': tf, 'backward_ms': tb, 'backward_over_forward': tb / tf, 'stages_ms': prof,
            'gpu_launches': launches, 'clocks': clocks}
        dyn.close()
        del dyn, x, J
        torch.cuda.empty_cache()
    except Exception as e:  # e.g. the tapes do not fit
        out['error'] = repr(e)[:300]
    torch.cuda.empty_cache()
    if args.no_fdcheck:
        return out
    # differentiation case: finite-difference check and timing
    def fd_check(dyn, x, final_theta, mask, gen, eps_list):
        grad = torch.cat([xx.grad.flatten() for xx in x])
        fd = []
        for eps in eps_list:
            for _ in range(8):
                d = torch.randn(grad.numel(), generator=gen, dtype=torch.float64).cuda()
                d /= d.norm()
                parts = torch.split(d, [xx.numel() for xx in x])
                with torch.no_grad():
                    tp = final_theta([(xx + eps * q.view_as(xx)).detach() for xx, q in zip(x, parts)])
                    tm = final_theta([(xx - eps * q.view_as(xx)).detach() for xx, q in zip(x, parts)])
                    # J(x + eps d) - J(x - eps d) summed as mask (tp - tm)(tp + tm): no cancellation of two 1e9 sums
                    fdv = (mask * (tp - tm) * (tp + tm)).sum().item() / (2 * eps)
                ad = torch.dot(grad, d).item()
                fd.append({'eps': eps, 'adjoint': ad, 'central_difference': fdv,
                           'rel_diff': abs(fdv - ad) / max(abs(ad), 1e-300)})
        # |FD - AD| over the RMS of the sampled directional derivatives: the
        # error on the scale of a typical direction (a direction whose
        # derivative happens to be small inflates its own rel_diff)
        def on_rms(e):
            sel = [f for f in fd if f['eps'] == e]
            rms = (sum(f['adjoint'] ** 2 for f in sel) / len(sel)) ** .5
            return max(abs(f['central_difference'] - f['adjoint']) for f in sel) / max(rms, 1e-300)
        return {'directions_per_eps': 8,
                'max_rel_diff': {str(e): max(f['rel_diff'] for f in fd if f['eps'] == e) for e in eps_list},
                'max_abs_diff_over_rms': {str(e): on_rms(e) for e in eps_list},
                'per_direction': fd}

    st4 = ic.config(4)
    dyn, x, final_theta, mask, J, (tf, tb, prof4, launches, clocks) = timed(st4, st4.nsteps, st4.remap_every, 5, 1)
    gen = torch.Generator(device='cpu').manual_seed(4)
    fd_spec = fd_check(dyn, x, final_theta, mask, gen, (1e-6, 1e-3))
    dyn.close()
    torch.cuda.empty_cache()
    # the same case with the exact ties of its initial state broken (uniform
    # dp, x-independent winds, v = 0 make the limiters non-differentiable
    # there): 0.01 Pa, 1e-4 K and 1e-3 m/s of seeded noise
    st4n = ic.config(4)
    rng = np.random.default_rng(40)
    st4n.dp = st4n.dp + rng.normal(0, 0.01, st4n.dp.shape)
    st4n.pt = st4n.pt + rng.normal(0, 1e-4 / P0K, st4n.pt.shape)
    st4n.u = st4n.u + rng.normal(0, 1e-3, st4n.u.shape)
    st4n.v = st4n.v + rng.normal(0, 1e-3, st4n.v.shape)
    dyn, x, final_theta, mask, _, _ = timed(st4n, st4n.nsteps, st4n.remap_every, 5, 0)
    fd_generic = fd_check(dyn, x, final_theta, mask, gen, (1e-6,))
    out['differentiation_case'] = {
        'workload': 'jet 512x512x32 (seed 2), 20 steps, dt 30 s, remap every 5, checkpoints every 5',
        'J': J.item(), 'forward_ms': tf, 'backward_ms': tb, 'backward_over_forward': tb / tf, 'stages_ms': prof4,
        'cell_steps_per_s': st4.cells * st4.nsteps / ((tf + tb) * 1e-3),
        'fd_check': fd_spec,
        'fd_check_ties_broken': fd_generic,
        'clocks': clocks,
    }
    dyn.close()
    torch.cuda.empty_cache()
    return out


def ensemble_leg(args, torch):
    """The batched ensemble: 64 members of uneven sizes (grids from
    {64, 128, 256, 512}^2, layers from {20, 32, 48, 64}, bubble or jet,
    seed 3), mixed form, remap every 5 steps, 100 steps: as one launch of
    the persistent kernel captured in a CUDA graph (strip heights autotuned
    per grid size), as the per-member kernels captured over 8 streams in
    one graph, and launching the members one by one on one stream; then the
    gradient of J = sum(mask theta^2) of 8 members (FP64 form, 20 steps,
    checkpoints every 5)."""
    from atmdyn import ic
    from atmdyn.ensemble import Ensemble
    from atmdyn.adjoint import integrate, gaussian_mask
    from atmdyn import Dycore
    members = ic.ensemble_members(64, seed=3)
    out = {'members': len(members), 'cells': sum(st.cells for st in members),
           'workload': '64 members, grids {64..512}^2 x {20..64} layers, bubble or jet (seed 3), mixed form, '
                       'remap every 5 steps, 100 steps'}
    nsteps = 100
    # one stream, member after member
    ens = Ensemble(members, 'mixed', nstreams=1)
    ens.step_eager(5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ens.step_eager(10)
    torch.cuda.synchronize()
    t_seq = (time.perf_counter() - t0) / 10
    ens.close()
    del ens
    torch.cuda.empty_cache()
    # the 100 steps as one graph over 8 streams, one launch
    ens = Ensemble(members, 'mixed', nstreams=8)
    ens.step_eager(5)
    t0 = time.perf_counter()
    ens.capture(5, cycles=nsteps // 5)
    t_cap = time.perf_counter() - t0
    ens.replay(1)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.replay(1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    steps = ens.cycle
    out['graph'] = {'cell_steps_per_s': out['cells'] * steps / (ms * 1e-3), 'ms_per_step': ms / steps,
                    'steps': steps, 'streams': 8, 'graph_launches': 1, 'capture_s': t_cap,
                    'stable': ens.stable()}
    out['one_stream_eager'] = {'cell_steps_per_s': out['cells'] / t_seq, 'ms_per_step': 1e3 * t_seq}
    out['graph_speedup'] = out['graph']['cell_steps_per_s'] / out['one_stream_eager']['cell_steps_per_s']
    ens.close()
    del ens
    torch.cuda.empty_cache()
    # the persistent kernel: strip heights autotuned per grid size, then the
    # 100 steps as ONE cooperative launch captured in a CUDA graph
    ens = Ensemble(members, 'mixed', nstreams=1)
    ens.step_eager(5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    table = ens.autotune(steps=2, reps=2)
    t_tune = time.perf_counter() - t0
    ens.capture_persistent(5, cycles=nsteps // 5)
    ens.replay(1)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.replay(1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out['persistent'] = {'cell_steps_per_s': out['cells'] * nsteps / (ms * 1e-3), 'ms_per_step': ms / nsteps,
                         'steps': nsteps, 'kernel_launches': 1, 'graph_launches': 1,
                         'strip_rows_by_grid': {str(k): v for k, v in sorted(table.items())},
                         'autotune_s': t_tune, 'barrier_timed_out': ens.barrier_timed_out(),
                         'stable': ens.stable()}
    out['persistent_speedup_vs_stream_graph'] = out['persistent']['cell_steps_per_s'] / out['graph']['cell_steps_per_s']
    ens.close()
    del ens
    torch.cuda.empty_cache()
    # adjoint on 8 members
    adj = []
    t0 = time.perf_counter()
    for st in members[:8]:
        dyn = Dycore(st)
        dyn.adj_enable()
        mask = gaussian_mask(st, min(300e3, 0.2 * st.nx * st.dx), device='cuda')
        x = [torch.tensor(np.ascontiguousarray(a), device='cuda', requires_grad=True)
             for a in (st.dp, st.pt, st.u, st.v)]
        y = integrate(dyn, x, 20, st.dt, st.remap_every, 5)
        J = (mask * (y[1] * P0K) ** 2).sum()
        J.backward()
        gn = float(sum(xx.grad.norm() ** 2 for xx in x) ** 0.5)
        adj.append({'member': st.name, 'nx': st.nx, 'nlay': st.nlay, 'J': J.item(), 'grad_norm': gn,
                    'finite': bool(np.isfinite(gn))})
        dyn.close()
    torch.cuda.synchronize()
    out['adjoint_members'] = {'count': 8, 'steps': 20, 'checkpoint_every': 5, 'wall_s': time.perf_counter() - t0,
                              'members': adj}
    return out


def e2e_runs(dy, st, K, stream, torch, max_over_ranks, world):
    """End to end through the C ABI with host buffers.

    e2e: every step uploads the four prognostic fields from pinned host
    memory (the reference's host arrays), runs the step and downloads them
    with the stability flag -- the drop-in used from a host time loop that
    keeps its state in host arrays.
    e2e_resident: the state is uploaded from pinned host memory before the
    first step and downloaded after the last, inside the timed region, with
    the stability flag read back every step."""
    from atmdyn.dycore import with_halo, HALO
    from atmdyn._lib import ATM_DP, ATM_PT, ATM_UD, ATM_VD
    fields = (ATM_DP, ATM_PT, ATM_UD, ATM_VD)
    shape = (st.nlay, st.ny + 2 * HALO, st.nx + 2 * HALO)
    host = [torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for _ in fields]
    for h, f in zip(host, fields):
        dy.get_into(f, h)
    nbytes = sum(h.nbytes for h in host)
    cells = st.cells
    out = []
    for mode in ('roundtrip', 'resident'):
        Ke = max(2, min(K, 6)) if mode == 'roundtrip' else K
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        if mode == 'resident':
            for h, f in zip(host, fields):
                dy.upload(f, h)
        for s in range(Ke):
            if mode == 'roundtrip':
                for h, f in zip(host, fields):
                    dy.upload(f, h)
            dy.step(DT, remap=((s + 1) % REMAP_EVERY == 0), check_stable=True)
            if mode == 'roundtrip':
                for h, f in zip(host, fields):
                    dy.get_into(f, h)
        if mode == 'resident':
            for h, f in zip(host, fields):
                dy.get_into(f, h)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1))
        v = world * cells * Ke / (ms * 1e-3)
        if mode == 'roundtrip':
            out.append({'value': v, 'unit': 'cell-steps/s', 'h2d_bytes_per_step': nbytes,
                        'd2h_bytes_per_step': nbytes + 4, 'steps': Ke,
                        'how': 'per step: upload dp/pt/ud/vd from pinned host, atm_step, download + stability flag'})
        else:
            out.append({'value': v, 'unit': 'cell-steps/s', 'h2d_bytes_per_step': nbytes / Ke,
                        'd2h_bytes_per_step': nbytes / Ke + 4, 'steps': Ke,
                        'how': 'state uploaded before step 1 and downloaded after step K inside the timed region'})
    return out[0], out[1]


def probe_remap_adjoint(args):
    """A small case for ncu captures of the remap adjoint kernels (nothing
    is timed here): a jet at nx x nx x nlay, two forward steps, then three
    calls of the remap adjoint with a dense seeded output adjoint."""
    import torch
    torch.cuda.set_device(0)
    from atmdyn import ic, Dycore
    from atmdyn.dycore import HALO
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    g = Dycore(st)
    for _ in range(2):
        g.step(DT, remap=False, check_stable=False)
    g.adj_enable()
    rng = np.random.default_rng(7)
    shape = (st.nlay, st.ny + 2 * HALO, st.nx + 2 * HALO)
    for n in ('dp', 'pt', 'ud', 'vd'):
        g.adj_set('out', n, rng.normal(0, 1, shape))
    for _ in range(3):
        g.adj_remap()
    g.sync()
    g.close()
    print('remap adjoint probe done: %dx%dx%d' % (args.nx, args.nx, args.nlay))


def probe_steps(args):
    """A small case for ncu captures of the step kernels (nothing is timed
    here): the forward forms, or the forward + adjoint of the headline loss."""
    import torch
    torch.cuda.set_device(0)
    from atmdyn import ic, Dycore
    st = ic.jet_case(args.nx, args.nx, args.nlay, 25e3, 25e3, seed=0)
    if args.probe == 'forward':
        for form in args.forms.split(','):
            dy = Dycore(st, form)
            for n in range(args.warmup + args.steps):
                dy.step(DT, remap=(n + 1) % REMAP_EVERY == 0, check_stable=False)
            assert dy.check_stability()
            dy.close()
    else:
        from atmdyn.adjoint import integrate
        dyn = Dycore(st)
        dyn.adj_enable()
        x = [torch.tensor(np.ascontiguousarray(a), device='cuda', requires_grad=True)
             for a in (st.dp, st.pt, st.u, st.v)]
        y = integrate(dyn, x, args.steps, DT, REMAP_EVERY, ADJ_CKPT)
        ((y[1] * P0K) ** 2).sum().backward()
        torch.cuda.synchronize()
        dyn.close()
    print('probe done: %s %dx%dx%d' % (args.probe, args.nx, args.nx, args.nlay))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=16)
    ap.add_argument('--warmup', type=int, default=8)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline leg')
    ap.add_argument('--nx', type=int, default=NX, help='grid size (profiling runs use smaller cases)')
    ap.add_argument('--nlay', type=int, default=NLAY)
    ap.add_argument('--forms', default='fp64,mixed')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-adjoint', action='store_true',
                    help='skip the masked-loss and differentiation-case legs of the adjoint')
    ap.add_argument('--no-ensemble', action='store_true', help='skip the batched-ensemble leg')
    ap.add_argument('--no-fdcheck', action='store_true', help='skip the differentiation case of the adjoint leg')
    ap.add_argument('--no-physics', action='store_true', help='skip the column-physics leg')
    ap.add_argument('--no-radiation', action='store_true', help='skip the radiation leg')
    ap.add_argument('--probe', choices=['remap_adj', 'forward', 'adjoint', 'radiation'], default=None,
                    help='profiling case instead of the benchmark, on a jet at --nx x --nx x --nlay: remap_adj = '
                         'two steps, then three calls of the remap adjoint with a dense random output adjoint; '
                         'forward = --warmup + --steps steps of each form in --forms (remap every 8); adjoint = '
                         '--steps steps forward + adjoint of J = sum(theta^2) (checkpoints every 8); radiation = '
                         'three calls of the radiation')
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.probe == 'remap_adj':
        probe_remap_adjoint(args)
        return
    if args.probe == 'radiation':
        probe_radiation(args)
        return
    if args.probe in ('forward', 'adjoint'):
        probe_steps(args)
        return
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
