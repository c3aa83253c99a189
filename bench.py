#!/usr/bin/env python
"""Throughput benchmark of the B200 em2d time step.

Workload: the uniform warm plasma -- 2048x2048 cells, dx = dy = 0.1,
dt = 0.07, periodic, 16x16 tiles, one electron species with 8x8 particles
per cell (268,435,456 particles), density 1, UDistribution::Thermal
uth = 0.05 (the reference's own seeded generator), ufl = 0, FP32.  A step is
one Simulation::advance (push + move/deposit + sort + current guard cells +
Yee).  Metric: particle pushes per second (sum of particles moved per step,
as Simulation::get_nmove counts them, divided by the step time).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (launched by torchrun) every rank runs its own replica of the
workload (a single run is not decomposed across GPUs; ensembles shard by
run) and the timing is the maximum over ranks.  ``--impl reference`` times the reference's own OpenMP
build (oracle/_ref, AVX2 variant) on the host cores instead.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, 'zpic-parallel_b200'), os.path.join(ROOT, 'oracle')):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# workload (uniform warm plasma)
NCELL = 2048
TILE = 16
PPC = 8
UTH = 0.05
DT = 0.07
DX = 0.1
METRIC = 'particle_pushes_per_second'
UNIT = 'pushes/s'
# algorithmic bytes (reference state layout): 56 B per particle push
# (int2 cell + float2 position + float3 momentum, read and written); the
# particle kernel also reads E and B (24 B/cell) and writes J (12 B/cell)
BYTES_PER_PUSH = 56
PARTICLE_KERNEL_BYTES_PER_CELL = 36
# the whole step's algorithmic bytes per cell: the particle kernel's 36 plus
# the Yee solve (read E, B, J: 36 B; write E, B: 24 B)
STEP_BYTES_PER_CELL = 96
# steady-state timing: after this many steps of the run, over this many steps
# (a whole period of the library's in-tile reorder, so that the figure is its
# average over a period, not a window that happens to follow a reorder)
STEADY_AFTER = 100
STEADY_STEPS = 50
# the batched Weibel ensemble: runs and steps of the workload
ENSEMBLE_RUNS = 256
ENSEMBLE_STEPS = 500


def workload_config(ncell=NCELL):
    return {
        'workload': 'uniform warm plasma %dx%d cells, 16x16 tiles, 8x8 ppc, uth 0.05, periodic' % (ncell, ncell),
        'cells': ncell * ncell, 'particles': ncell * ncell * PPC * PPC, 'tile': [TILE, TILE],
        'dx': DX, 'dt': DT, 'species': 1,
        'current_accumulation': 'fixed point in shared memory (option jacc 2, default)',
        'l2': 'inputs larger than L2 (particle state %.1f GB)' % (ncell * ncell * PPC * PPC * 24 / 1e9),
    }


def peaks():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def ncu_traffic_per_particle():
    """DRAM bytes per particle of the particle kernel from the committed ncu summary."""
    p = os.path.join(ROOT, 'profiles', 'particles_uniform_plasma.md')
    if not os.path.exists(p):
        return None
    m = re.search(r'dram_bytes_per_particle:\s*([0-9.]+)', open(p).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed
    region: the sampler is started and its first sample awaited before the
    region begins, and only samples that arrive inside it are kept (the one
    nearest to it when the region is shorter than the sampling period)."""

    def __init__(self, index, period_ms=25):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.lines = []                       # (arrival time, csv line)
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index),
                 '--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
                 'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
                 'clocks_event_reasons.sw_power_cap',
                 '--format=csv,noheader,nounits', '-lms', str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 2.0
            while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
        except (OSError, FileNotFoundError):
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def __exit__(self, *a):
        self.t1 = time.perf_counter()
        if self.proc:
            time.sleep(2 * self.period_ms / 1e3)      # the samples still in the pipe
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        slack = 2 * self.period_ms / 1e3
        inside = [ln for ts, ln in self.lines if self.t0 is not None and self.t0 <= ts <= self.t1 + slack]
        if not inside and self.lines and self.t0 is not None:
            inside = [min(self.lines, key=lambda e: abs(e[0] - self.t0))[1]]
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in inside:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[3 + k].lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': mx,
                'reasons': sorted(reasons), 'samples': len(sm)}


def dist_setup(args):
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = 'nccl' if torch.cuda.is_available() else 'gloo'
        if backend == 'nccl':
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = 'cuda' if torch.cuda.is_available() else 'cpu'
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU reference arm: the reference's own OpenMP build (oracle/_ref)
# ---------------------------------------------------------------------------
def reference_sample(ncell, steps, warmup, threads=None):
    from em2d_oracle import RefSim, ref_available
    variant = 'avx2' if ref_available('avx2') else 'scalar'
    nt = ncell // TILE
    s = RefSim((nt, nt), (TILE, TILE), (ncell * DX, ncell * DX), DT, variant=variant,
               threads=threads or os.cpu_count())
    s.add_species(-1.0, (PPC, PPC), udist=('thermal', (UTH, UTH, UTH), (0, 0, 0)))
    s.advance(warmup)
    n0 = s.nmove()
    t0 = time.perf_counter()
    s.advance(steps)
    dt = time.perf_counter() - t0
    pushes = s.nmove() - n0
    cores = s.threads
    s.close()
    return pushes / dt, dt / steps, cores, variant


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    from em2d_oracle import ref_available
    if not ref_available('scalar') and not ref_available('avx2'):
        print(json.dumps({'impl': 'reference', 'unavailable': 'reference build oracle/_ref missing'}))
        return 0
    # the workload itself (2048^2 cells, 268 M particles: ~8 GB of host
    # memory, ~0.4 s per step on 16 cores) unless a smaller box is asked for
    ncell = args.reference_cells
    rate, tstep, cores, variant = reference_sample(ncell, args.steps, args.warmup)
    cfg = workload_config(ncell)
    line = {
        'metric': METRIC, 'value': rate, 'unit': UNIT, 'impl': 'reference',
        'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': tstep * 1e3, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (reference RNG, seeded)',
        'config': cfg,
        'cpu_baseline': {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
                         'sample': '%dx%d cells (%d particles), openmp/em2d %s build, %d threads, '
                                   '%d steps after %d untimed, step loop timed'
                                   % (ncell, ncell, ncell * ncell * PPC * PPC, variant, cores,
                                      args.steps, args.warmup)},
        'e2e': {'value': rate, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def apply_options(s, args):
    """Library options given on the command line (default: the library's)."""
    if getattr(args, 'reorder', None) is not None:
        s.set_option('reorder', args.reorder)
    return s


def capacity_option(s, args):
    """Library option set before species are added (their initial capacity)."""
    if getattr(args, 'capacity_factor', None) is not None:
        s.set_option('capacity_factor', args.capacity_factor)
    return s


def make_sim(zb, ncell, device, args=None):
    nt = ncell // TILE
    s = zb.Simulation((nt, nt), (TILE, TILE), (ncell * DX, ncell * DX), DT, device=device)
    s.add_species(-1.0, (PPC, PPC), udist=('thermal', (UTH, UTH, UTH), (0, 0, 0)))
    return apply_options(s, args)


def run_gpu(args, world, rank, local):
    import numpy as np
    import torch
    import zpic_b200 as zb

    torch.cuda.set_device(local)
    ncell = args.cells
    sim = make_sim(zb, ncell, local, args)
    np_total = sim.np_total(0)
    stream = torch.cuda.ExternalStream(sim.stream_handle(), device=local)

    # per-phase CUDA events as nodes of the step graph (library option
    # profile 2), so that the particle kernel is timed inside the timed region
    sim.set_option('profile', 2)
    # warm-up (also captures the CUDA graph of one step)
    sim.advance(args.warmup)
    sim.synchronize()
    sim.reset_phase_times()

    # ---- device-timed region: K steps, inputs resident in HBM ----
    l0 = sim.launch_count()
    n0 = sim.nmove()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sim.advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    t_ms = ev0.elapsed_time(ev1)
    launches = sim.launch_count() - l0
    pushes = sim.nmove() - n0
    t_max = max_over_ranks(t_ms, world)
    value = pushes * world / (t_max / 1e3)

    # ---- per-kernel timing: the particle kernel's events in the same K steps;
    # the other phases from K more steps issued eagerly with events around
    # every phase (a breakdown only) ----
    part_ms, part_n = sim.phase_times()['particles']
    sim.set_option('profile', 1)
    sim.reset_phase_times()
    sim.advance(args.steps)
    sim.synchronize()
    ph = sim.phase_times()
    # ---- steady state: the same timing once the run is past 100 steps (the
    # particles' in-tile order has decayed, as in the workload's 100-step runs) ----
    sim.set_option('profile', 2)
    done = args.warmup + 2 * args.steps
    sim.advance(max(0, STEADY_AFTER - done))
    sim.synchronize()
    sim.reset_phase_times()
    s0, m0 = sim.iter(), sim.nmove()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    w0.record(stream)
    sim.advance(STEADY_STEPS)
    w1.record(stream)
    w1.synchronize()
    ts = max_over_ranks(w0.elapsed_time(w1), world)
    sp_ms, sp_n = sim.phase_times()['particles']
    steady = {'after_steps': s0, 'steps': STEADY_STEPS, 'ms_per_step': ts / STEADY_STEPS,
              'value': (sim.nmove() - m0) * world / (ts / 1e3), 'unit': UNIT,
              'particle_launch_ms': sp_ms / max(1, sp_n)}
    sim.set_option('profile', 0)
    sim.set_option('graph', 1)
    per_launch_ms = part_ms / max(1, part_n)
    hbm, peak_kind = peaks()
    alg_bytes = BYTES_PER_PUSH * np_total + PARTICLE_KERNEL_BYTES_PER_CELL * ncell * ncell
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    steady['roofline_frac'] = alg_bytes / (steady['particle_launch_ms'] / 1e3) / 1e9 / hbm
    tpp = ncu_traffic_per_particle()
    roofline = {
        'kernel': 'k_particles (fused push, move, deposit, walls, leaver detection)',
        'bound': 'hbm', 'achieved': achieved, 'peak': hbm, 'unit': 'GB/s',
        'frac': achieved / hbm, 'peak_kind': peak_kind,
        'traffic': (tpp * np_total) if tpp else None,
        'algorithmic_bytes_per_launch': alg_bytes,
        'launch_ms': per_launch_ms,
        'phase_ms_per_step': {k: v[0] / args.steps for k, v in ph.items()},
        'phase_note': 'launch_ms: particle kernel timed by event nodes of the step graph during the timed steps; '
                      'phase_ms_per_step: the K steps after them, issued eagerly with events around every phase '
                      '(the sort and the current + field phases run side by side on two streams)',
    }

    # ---- end-to-end through the C-ABI with host buffers ----
    # timed: upload of the particle state from pinned host memory, K steps,
    # and the per-step energy diagnostics read back to the host (as
    # Simulation::energy_info does)
    npt, ix, x, u = sim.particles(0)
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    ix, x, u, npt = pin(ix), pin(x), pin(u), pin(npt)
    h2d = ix.nbytes + x.nbytes + u.nbytes + npt.nbytes
    # one untimed upload first (as the warm-up steps are untimed): the first
    # DMA from freshly pinned pages runs at ~45 instead of ~55 GB/s
    sim.set_particles(0, npt, ix, x, u)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.set_particles(0, npt, ix, x, u)
    for _ in range(args.steps):
        sim.advance(1)
        sim.species_energy(0)
        sim.emf_energy()
    sim.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = np_total * args.steps * world / e2e_s
    # species energy (1 double) + per-tile field energy partials (6 doubles per
    # tile, summed on the host in tile order as EMF::get_energy does)
    d2h = 8 + 6 * 8 * (ncell // TILE) ** 2
    sim.close()

    # ---- chosen vs plain: the same workload and timing with the plain FP32
    # tile current (FP32 shared-memory atomics, the reference's FP32 sums in
    # another order; option jacc 0) ----
    psim = make_sim(zb, ncell, local, args)
    psim.set_option('jacc', 0)
    pstream = torch.cuda.ExternalStream(psim.stream_handle(), device=local)
    psim.advance(args.warmup)
    psim.synchronize()
    pn0 = psim.nmove()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    q0.record(pstream)
    psim.advance(args.steps)
    q1.record(pstream)
    q1.synchronize()
    tp = max_over_ranks(q0.elapsed_time(q1), world)
    plain = {'value': (psim.nmove() - pn0) * world / (tp / 1e3), 'unit': UNIT, 'ms_per_step': tp / args.steps,
             'how': 'same steps with FP32 shared-memory atomics for the tile current (option jacc 0) '
                    'instead of the fixed-point accumulation'}
    psim.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from em2d_oracle import ref_available
            if ref_available('avx2') or ref_available('scalar'):
                rate, tstep, cores, variant = reference_sample(args.ref_cells, args.ref_steps, 1)
                cpu = {'value': rate, 'unit': UNIT, 'cores': cores, 'kind': 'reference',
                       'sample': '%dx%d cells of the workload (%d particles), openmp/em2d %s build, '
                                 '%d steps, step loop timed' % (args.ref_cells, args.ref_cells,
                                                                args.ref_cells ** 2 * PPC * PPC, variant,
                                                                args.ref_steps)}
        except Exception as e:  # reported, not fatal
            cpu = {'value': None, 'error': str(e)}

    # ---- the ensemble half of the metric: batched vs plain run-steps/s on
    # the 256-run Weibel ensemble, its own 500 steps whatever --steps says ----
    ens = None
    if not args.no_ensemble:
        ens = ensemble_measure(args, world, rank, local, ENSEMBLE_RUNS, ENSEMBLE_STEPS)

    clocks = clk.summary()
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t_max / args.steps,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32', 'data': 'synthetic (reference RNG, seeded Thermal uth 0.05)',
            'config': workload_config(ncell),
            'roofline': roofline,
            'step_roofline': {
                'bytes_per_step': BYTES_PER_PUSH * np_total + STEP_BYTES_PER_CELL * ncell * ncell,
                'achieved': (BYTES_PER_PUSH * np_total + STEP_BYTES_PER_CELL * ncell * ncell) / (t_max / args.steps / 1e3) / 1e9,
                'unit': 'GB/s',
                'frac': (BYTES_PER_PUSH * np_total + STEP_BYTES_PER_CELL * ncell * ncell) / (t_max / args.steps / 1e3) / 1e9 / hbm,
                'note': 'whole step (56 B per particle push + 96 B per cell) over the timed step time'},
            'cpu_baseline': cpu,
            'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': h2d / args.steps,
                    'd2h_bytes_per_step': d2h,
                    'note': 'particle state uploaded once from pinned host memory inside the timed '
                            'region (bytes amortised over the K steps), energies read back every step'},
            'gpu_launches': launches,
            'clocks': clocks,
            'cell_updates_per_second': ncell * ncell * args.steps * world / (t_max / 1e3),
            'plain': plain,
            'chosen_over_plain': value / plain['value'],
            'steady_state': steady,
        }
        if ens is not None:
            line['ensemble'] = ens
        print(json.dumps(line))
    return 0


def ensemble_specs(nruns, seed=0):
    """Batched Weibel ensemble: grid N x N with N in {64,...,512}, ppc in
    {2x2, 4x4, 8x8}, |ufl_z| ~ U[0.2, 0.8], uth ~ U[0.02, 0.15], drawn from a
    seeded PCG64 generator."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = [64, 96, 128, 192, 256, 384, 512]
    out = []
    for _ in range(nruns):
        n = int(rng.choice(sizes))
        p = int(rng.choice([2, 4, 8]))
        uz = float(rng.uniform(0.2, 0.8))
        uth = float(rng.uniform(0.02, 0.15))
        out.append((n, p, uz, uth))
    return out


def ensemble_measure(args, world, rank, local, nruns, steps):
    """Weibel ensemble: many independent runs advanced together (one launch
    per phase over all runs, CUDA-graph replay) vs the same runs each advanced
    through its own graph, one after another and all at once on separate
    streams.  Metric: aggregate run-steps per second, timed on the device.
    Returns the measurement as a dict (rank 0), None elsewhere."""
    import torch
    import zpic_b200 as zb
    torch.cuda.set_device(local)
    specs = ensemble_specs(nruns)
    specs = specs[rank::world]                  # runs shard across ranks, no exchange
    sims = []
    h0 = time.perf_counter()
    for n, p, uz, uth in specs:
        s = capacity_option(zb.Simulation((n // TILE, n // TILE), (TILE, TILE), (n * DX, n * DX), DT, device=local),
                            args)
        s.add_species(-1.0, (p, p), udist=('thermalcorr', (uth, uth, uth), (0, 0, uz)))
        s.add_species(1.0, (p, p), udist=('thermalcorr', (uth, uth, uth), (0, 0, -uz)))
        sims.append(apply_options(s, args))
    setup_s = time.perf_counter() - h0
    nparticles = sum(s.np_total(0) + s.np_total(1) for s in sims)
    batch = zb.Batch(sims)
    # device timing: events on one stream that every participating stream
    # joins before and after the timed region
    clock = torch.cuda.Stream()
    bstream = torch.cuda.ExternalStream(batch.stream_handle())
    sstreams = [torch.cuda.ExternalStream(s.stream_handle()) for s in sims]

    def timed(streams, work):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(clock)
        for st in streams:
            st.wait_event(ev0)
        work()
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            clock.wait_event(e)
        ev1.record(clock)
        torch.cuda.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1) * 1e-3, world)

    chunks = batch.autotune(2) if args.autotune else None
    batch.advance(args.warmup)
    batch.synchronize()
    l0 = batch.launch_count()
    with ClockSampler(local) as clk:
        tb = timed([bstream], lambda: batch.advance(steps))
    batch.synchronize()
    launches = batch.launch_count() - l0
    # plain: each run advanced on its own through its own CUDA graph, the runs
    # one after another on the device (a sweep run by run) ...
    for s in sims:
        s.advance(args.warmup)
    for s in sims:
        s.synchronize()

    def serial():
        prev = None
        for s, st in zip(sims, sstreams):
            if prev is not None:
                st.wait_event(prev)
            s.advance(steps)
            prev = torch.cuda.Event()
            prev.record(st)
    tp = timed(sstreams, serial)
    for s in sims:
        s.synchronize()

    # ... and all runs issued at once on their own streams
    def concurrent():
        for s in sims:
            s.advance(steps)
    tc = timed(sstreams, concurrent)
    for s in sims:
        s.synchronize()
    # tile-slot rebuilds over the three timed runs (and warm-ups)
    repacks = sum(s.repacks(k) for s in sims for k in range(2))
    relocations = sum(s.relocations(k) for s in sims for k in range(2))
    batch.close()
    for s in sims:
        s.close()
    if rank != 0:
        return None
    return {
        'metric': 'ensemble_run_steps_per_second', 'value': nruns * steps / tb,
        'unit': 'run-steps/s', 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': tb / steps * 1e3,
        'config': {'workload': 'Weibel ensemble, %d runs (seeded PCG64 draw of N, ppc, ufl, uth), '
                               '%d steps' % (nruns, steps),
                   'particles_per_rank': nparticles, 'runs_per_rank': len(sims)},
        'plain': {'value': nruns * steps / tp, 'unit': 'run-steps/s',
                  'how': 'each run through its own CUDA graph, runs one after another'},
        'plain_concurrent': {'value': nruns * steps / tc, 'unit': 'run-steps/s',
                             'how': 'each run through its own CUDA graph on its own stream, all issued at once'},
        'batched_over_plain': tp / tb,
        'batched_over_plain_concurrent': tc / tb,
        'pushes_per_second': nparticles * world * steps / tb,
        'gpu_launches': launches,
        'ctas_per_tile': chunks if chunks is not None else 'automatic',
        'setup_s': setup_s,
        'slot_repacks': repacks, 'tiles_relocated': relocations,
        'clocks': clk.summary(),
    }


def run_ensemble(args, world, rank, local):
    steps = args.steps if args.steps_given else ENSEMBLE_STEPS
    ens = ensemble_measure(args, world, rank, local, args.runs, steps)
    if rank == 0:
        line = dict(ens)
        line.update({'n_gpus': world, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
                     'dtype': 'f32', 'data': 'synthetic (reference RNG, seeded)'})
        print(json.dumps(line))
    return 0


def run_lwfa(args, world, rank, local):
    """Laser wakefield with a moving window: 4096x512 cells, dx 0.025, dy 0.1,
    dt 0.022, 16x16 tiles, electrons 4x2 ppc behind a density step at x = 20,
    cold; Gaussian pulse a0 2, omega0 10, W0 4, fwhm 2 (start 17, focus 20,
    axis 25.6, Ez polarisation); no current filter.  Every step is one
    Simulation::advance_mov_window from t = 0 (the window moves 0.88 cells per
    step, injecting a new column at the right edge).  Metric: particle pushes
    per second over the whole run, timed on the device."""
    import torch
    import zpic_b200 as zb
    torch.cuda.set_device(local)
    nx, ny = 4096, 512
    t_set0 = time.perf_counter()
    s = zb.Simulation((nx // TILE, ny // TILE), (TILE, TILE), (nx * 0.025, ny * 0.1), 0.022, device=local)
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 20.0, 0))
    s.synchronize()
    t_set1 = time.perf_counter()
    # the Gaussian pulse is computed on the host (libm cos/exp/atan2, so that
    # the fields match the reference's bit for bit) and uploaded
    s.add_laser('gaussian', start=17.0, fwhm=2.0, a0=2.0, omega0=10.0, W0=4.0, focus=20.0, axis=25.6, sin_pol=1)
    s.synchronize()
    t_set2 = time.perf_counter()
    s.set_moving_window()
    apply_options(s, args)
    np0 = s.np_total(0)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)
    steps = args.steps if args.steps_given else 2000
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    l0, n0 = s.launch_count(), s.nmove()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        h0 = time.perf_counter()
        s.advance_mov_window(steps)
        host_s = time.perf_counter() - h0       # time the host takes to issue the steps
        ev1.record(stream)
        ev1.synchronize()
    t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)
    pushes = s.nmove() - n0
    e, b = s.emf_energy()
    # per-phase device time over 100 further steps (CUDA events around each phase)
    s.set_option('profile', 1)
    s.reset_phase_times()
    s.advance_mov_window(100)
    s.synchronize()
    phases = {k: v[0] / 100 for k, v in s.phase_times().items()}
    if rank == 0:
        print(json.dumps({
            'metric': METRIC, 'value': pushes * world / t, 'unit': UNIT, 'n_gpus': world,
            'steps': steps, 'warmup': 0, 'ms_per_step': t / steps * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic (step density, Gaussian laser, from t = 0)',
            'config': {'workload': 'laser wakefield, moving window, 4096x512 cells, 16x16 tiles, 4x2 ppc, '
                                   'a0 2, %d steps from t = 0' % steps,
                       'particles_initial': np0, 'particles_final': s.np_total(0)},
            'cell_updates_per_second': nx * ny * steps * world / t,
            'gpu_launches': s.launch_count() - l0,
            'field_energy_final': float(e.sum() + b.sum()),
            'phase_ms_per_step': phases,
            'host_issue_ms_per_step': host_s / steps * 1e3,
            'setup_s': {'simulation_and_species': t_set1 - t_set0, 'gaussian_laser_on_host': t_set2 - t_set1},
            'slot_repacks': s.repacks(0), 'tiles_relocated': s.relocations(0),
            'clocks': clk.summary(),
        }))
    s.close()
    return 0


def reference_cuda(ppc, ntiles, timeout=900):
    """The reference's own CUDA build (oracle/_ref/cuda/zpic, sm_100a) on its
    Weibel test: 32x32 tiles, two species, 500 steps.  Returns its printed
    GPart/s (host-timed around the step loop by the reference) or None."""
    exe = os.path.join(ROOT, 'oracle', '_ref', 'cuda', 'zpic')
    if not os.path.exists(exe):
        return None, 'reference CUDA build oracle/_ref/cuda/zpic missing'
    r = subprocess.run([exe, '-s', '-t', 'weibel', '-p', '%d,%d,%d,%d' % (ppc, ppc, ntiles, ntiles)],
                       capture_output=True, text=True, timeout=timeout)
    m = re.search(r'Performance:\s*([0-9.eE+-]+)\s*GPart/s', r.stdout)
    if r.returncode != 0 or not m:
        return None, 'reference run failed (rc %d): %s' % (r.returncode, (r.stdout + r.stderr)[-300:])
    return float(m.group(1)) * 1e9, r.stdout[-400:]


def run_weibel(args, world, rank, local):
    """Weibel instability at scale, the reference CUDA driver's own test
    (cuda/em2d/main.cpp:613-692): 32x32 tiles, ntiles x ntiles tiles, box
    0.1 per cell, dt 0.07, electrons and positrons 8x8 ppc ThermalCorr uth
    0.1, uz +-0.6, 500 steps.  Timed on the device; with --reference-gpu the
    reference's own CUDA build runs the same test on the same GPU."""
    import torch
    import zpic_b200 as zb
    torch.cuda.set_device(local)
    nt, ppc = args.weibel_tiles, 8
    steps = args.steps if args.steps_given else 500
    s = zb.Simulation((nt, nt), (32, 32), (nt * 32 * 0.1, nt * 32 * 0.1), 0.07, device=local)
    s.add_species(-1.0, (ppc, ppc), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)), name='electrons')
    s.add_species(1.0, (ppc, ppc), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)), name='positrons')
    # the plasma filaments (tiles reach twice the mean occupancy): CTAs in
    # proportion to each tile's particles
    s.set_option('chunks', -1)
    apply_options(s, args)
    npart = s.np_total(0) + s.np_total(1)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    n0 = s.nmove()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        s.advance(steps)
        ev1.record(stream)
        ev1.synchronize()
    t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)
    pushes = s.nmove() - n0
    s.close()
    ref = None
    if args.reference_gpu and rank == 0 and world == 1:
        rate, info = reference_cuda(ppc, nt)
        ref = {'value': rate, 'unit': UNIT, 'kind': 'reference CUDA build (cuda/em2d, sm_100a), same GPU',
               'timing': 'host timer around its 500-step loop', 'info': info}
    if rank == 0:
        print(json.dumps({
            'metric': METRIC, 'value': pushes * world / t, 'unit': UNIT, 'n_gpus': world,
            'steps': steps, 'warmup': 0, 'ms_per_step': t / steps * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic (reference RNG, seeded)',
            'config': {'workload': 'Weibel %dx%d cells, 32x32 tiles, 2 species x 8x8 ppc, %d steps'
                                   % (nt * 32, nt * 32, steps), 'particles': npart,
                       'ctas_per_tile': 'in proportion to tile occupancy (chunks -1)'},
            'reference_gpu': ref, 'clocks': clk.summary(),
        }))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--workload', default='plasma', choices=['plasma', 'ensemble', 'lwfa', 'weibel'])
    ap.add_argument('--weibel-tiles', type=int, default=64, help='weibel: tiles per side (32x32 cells each)')
    ap.add_argument('--reference-gpu', type=int, default=1, help='weibel: also run the reference CUDA build')
    ap.add_argument('--runs', type=int, default=256, help='ensemble runs (--workload ensemble)')
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--cells', type=int, default=NCELL, help='grid size (cells per side)')
    ap.add_argument('--ref-cells', type=int, default=512, help='cpu_baseline sample size (cells per side)')
    ap.add_argument('--reference-cells', type=int, default=NCELL,
                    help='--impl reference: grid size (cells per side; default the workload itself)')
    ap.add_argument('--ref-steps', type=int, default=10)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-ensemble', action='store_true', help='plasma workload only (skip the ensemble half)')
    ap.add_argument('--autotune', type=int, default=1, help='ensemble: autotune CTAs per tile first (1/0)')
    ap.add_argument('--capacity-factor', type=float, default=None,
                    help='ensemble: initial particle capacity per cell and ppc (library option "capacity_factor")')
    ap.add_argument('--reorder', type=int, default=None,
                    help='steps between in-tile particle reorders (library option "reorder"; default: the library default)')
    args = ap.parse_args()
    args.steps_given = any(a.startswith('--steps') for a in sys.argv[1:])
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args)
    try:
        if args.impl == 'reference':
            rc = run_reference(args, world, rank)
        elif args.workload == 'ensemble':
            rc = run_ensemble(args, world, rank, local)
        elif args.workload == 'lwfa':
            rc = run_lwfa(args, world, rank, local)
        elif args.workload == 'weibel':
            rc = run_weibel(args, world, rank, local)
        else:
            rc = run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == '__main__':
    sys.exit(main())
