#!/usr/bin/env python3
"""Benchmark of the B200 lattice Boltzmann engine on LBFlow's headline workload.

Workload (default): single-phase D3Q19 MRT in a synthetic porous cube of 256^3
voxels -- seeded N(0,1) noise, periodic Gaussian filter sigma = 3, threshold at
porosity 0.22, isolated fluid removed; fully periodic, tau = 1, g_x = 1e-5,
FP64 plain path.  A step is one stream-collide update of every fluid node.

Metric: fluid MLUPS (fluid nodes x steps / seconds / 1e6), the definition of
the reference's scripts/performance.py:80-85.  `value` is device-timed (CUDA
events on the engine's stream, inputs resident in HBM); `e2e` is the same
metric through the C ABI from host buffers (geometry upload, initialization,
every step's flux/mass read-back, final field download); `roofline` relates
the step kernel's algorithmic bytes to the measured HBM bandwidth.

    python bench.py [--steps K] [--warmup W] [--gpus N] [--storage fp64|fp32|fp16|bf16]
    python bench.py --impl reference      # the reference solver on the host cores
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'D3Q19 MRT fluid MLUPS (256^3 porous cube, porosity 0.22)'
# Algorithmic bytes per fluid-node update: read + write Q populations, plus
# the 4-byte link information (2*Q*s + 4).
ALG_BYTES = {'fp64': 2 * 19 * 8 + 4, 'fp32': 2 * 19 * 4 + 4, 'fp16': 2 * 19 * 2 + 4, 'bf16': 2 * 19 * 2 + 4,
             'bfp16': 2 * 19 * 2 + 2 + 4}
ELEM = {'fp64': 8, 'fp32': 4, 'fp16': 2, 'bf16': 2, 'bfp16': 2}


def measured_peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


def profile_traffic(storage):
    """DRAM bytes per step-kernel launch from the committed ncu summary, if any."""
    p = ROOT / 'profiles' / f'scsp_step_d3q19_mrt_{storage}_256.md'
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith('traffic_bytes_per_launch:'):
            v = line.split(':', 1)[1].strip()
            return None if v in ('', 'null') else float(v)
    return None


class ClockSampler:
    """SM clocks and throttle reasons sampled (NVML, read-only) during the timed region."""
    REASONS = {0x8: 'hw_slowdown', 0x40: 'hw_thermal_slowdown', 0x20: 'sw_thermal_slowdown',
               0x4: 'sw_power_cap', 0x80: 'hw_power_brake_slowdown'}

    def __init__(self, device, period=0.02):
        self.device = device
        self.period = period
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self._max = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._t = None
        return self

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.samples.append((sm, r, pw))
            except Exception:
                pass
            time.sleep(self.period)

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        reasons = set()
        for _, r, _ in self.samples:
            for bit, name in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        return {'sm_mhz': statistics.median(s[0] for s in self.samples), 'sm_max_mhz': self._max,
                'reasons': sorted(reasons), 'samples': len(self.samples),
                'power_w_max': max(s[2] for s in self.samples)}


def make_geometry(n, sigma, porosity, seed):
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((n, n, n), sigma=sigma, porosity=porosity, seed=seed)
    return np.where(fluid, 75, 255).astype(np.uint8)


LABELS = {75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}


def reference_run(workdir, geometry, steps, collision='MRT', grid_file=None):
    """Run the reference LBFlow binary once; return (fluid_nodes, steps, numerical seconds).
    Outputs go to workdir; field writes only at t = 0 (the reference always
    writes the initial fields), no checkpoint."""
    exe = ROOT / 'oracle' / '_ref' / 'LBFlow'
    nz, ny, nx = geometry.shape
    workdir.mkdir(parents=True, exist_ok=True)
    if grid_file is None:
        geometry.tofile(workdir / 'geometry.raw')
    else:
        (workdir / 'geometry.raw').symlink_to(grid_file)
    quiet = steps * 10
    prm = f'''gridFile "geometry.raw";
dimension {nz} {ny} {nx};
directions 19;
fileType "uint8";
latticeLen 1;
startTime 0;
endTime {steps};
writeInterval {quiet};
reportInterval {quiet};
restartInterval {quiet};
stopError 1e-6;
outPath "field";
logPath ".";
reportDir 0;
reportSlice 1 {nx - 2};
fluidModel "scsp";
equilModel "{collision}";
rexlationTime 1;
latticeSpeed 1;
alpha0 0.33333333333333331;
density 1;
contactAngle 90;
surfaceTension 0;
interfaceThickness 0.7;
75 "GV" "1e-5" "1" "0"
255 "SD" "90" "N/A" "N/A"
'''
    (workdir / 'input.prm').write_text(prm)
    r = subprocess.run([str(exe), 'input.prm'], cwd=workdir, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('reference run failed: ' + r.stdout[-500:])
    t = [json.loads(l[len('LBFlowTiming '):]) for l in r.stdout.splitlines() if l.startswith('LBFlowTiming ')][0]
    return t['fluid_nodes'], t['completed_steps'], t['numerical_seconds_max']


# Peak resident memory of one reference process on the 256^3 cube (measured:
# 13.6 GB; the reference builds per-voxel adjacency arrays), with headroom.
REF_BYTES_256 = 16e9


def host_memory_available():
    """Bytes this process may still use: MemAvailable, capped by a cgroup limit."""
    avail = None
    try:
        for line in open('/proc/meminfo'):
            if line.startswith('MemAvailable:'):
                avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    for path in ('/sys/fs/cgroup/memory.max', '/sys/fs/cgroup/memory/memory.limit_in_bytes'):
        try:
            lim = open(path).read().strip()
            used_p = path.replace('memory.max', 'memory.current').replace('limit_in_bytes', 'usage_in_bytes')
            if lim != 'max':
                used = int(open(used_p).read().strip())
                room = int(lim) - used
                avail = room if avail is None else min(avail, room)
            break
        except (OSError, ValueError):
            continue
    return avail


def host_cores():
    """Logical CPUs this process may run on, and physical cores (lscpu)."""
    try:
        logical = len(os.sched_getaffinity(0))
    except AttributeError:
        logical = os.cpu_count() or 1
    physical = None
    try:
        out = subprocess.run(['lscpu', '-p=CORE,SOCKET'], capture_output=True, text=True, timeout=10).stdout
        physical = len({l for l in out.splitlines() if l and not l.startswith('#')})
    except (OSError, subprocess.SubprocessError):
        pass
    return logical, physical


def reference_sample(steps, procs, size=256):
    """The reference solver on the benchmark's own workload: `procs`
    concurrent single-rank runs of the size^3 cube (sigma 3, porosity 0.22,
    seed 0 -- the geometry of the GPU arm), each `steps` steps after its
    initialization; aggregate fluid MLUPS = sum(fluid nodes x steps) / the
    slowest run's numerical seconds (scripts/performance.py:80-85)."""
    exe = ROOT / 'oracle' / '_ref' / 'LBFlow'
    if not exe.exists():
        return None, 'reference binary oracle/_ref/LBFlow is not built'
    g = make_geometry(size, 3.0, 0.22, 0)
    logical, physical = host_cores()
    with tempfile.TemporaryDirectory() as d:
        shared = Path(d) / 'geometry.raw'
        g.tofile(shared)
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(procs) as ex:
            res = list(ex.map(lambda k: reference_run(Path(d) / f'r{k}', g, steps, grid_file=shared), range(procs)))
    nodes = sum(r[0] * r[1] for r in res)
    secs = max(r[2] for r in res)
    return dict(value=nodes / secs / 1e6, unit='MLUPS', cores=procs, kind='reference',
                host_logical_cpus=logical, host_physical_cores=physical,
                sample=f'{procs} x reference LBFlow (1 rank each, no MPI on the host) on the {size}^3 cube of '
                       f'the benchmark (sigma 3, porosity 0.22, seed 0, {res[0][0]} fluid nodes), MRT FP64, '
                       f'{steps} steps each after initialization'), None


def reference_procs(limit=None):
    """Concurrent reference processes: one per logical CPU, as many as host
    memory holds at 16 GB each."""
    logical, _ = host_cores()
    avail = host_memory_available()
    by_mem = int(avail // REF_BYTES_256) if avail else 1
    n = max(1, min(logical, by_mem))
    return min(n, limit) if limit else n


def run_reference_arm(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    procs = reference_procs(limit=args.ref_procs)
    # A bounded sample of the workload: each process runs a few steps of the
    # full cube (about 6 s per step per core), so the arm ends in a few
    # minutes whatever --steps is.
    steps = max(1, min(args.steps + args.warmup, args.ref_steps))
    base, why = reference_sample(steps, procs)
    cfg = dict(workload='D3Q19 MRT single-phase porous cube 256^3, fp64 populations (reference solver)',
               nx=256, ny=256, nz=256, porosity=0.22, sigma=3, tau=1.0, g_x=1e-5, seed=0,
               parallelism=f'{procs} independent single-rank processes')
    if base is None:
        print(json.dumps({'impl': 'reference', 'unavailable': why}))
        return 0
    cfg['fluid_nodes'] = int(base['sample'].split(' fluid nodes')[0].rsplit(' ', 1)[-1])
    line = dict(impl='reference', metric=METRIC, value=base['value'], unit='MLUPS', n_gpus=args.gpus,
                steps=args.steps, warmup=args.warmup, ms_per_step=None, higher_is_better=True,
                scaling='weak', vs_baseline=None, dtype='f64', data='synthetic', config=cfg,
                cpu_baseline=base, e2e=dict(value=base['value'], unit='MLUPS', h2d_bytes_per_step=0,
                                            d2h_bytes_per_step=0))
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5000)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=('ours', 'reference'))
    ap.add_argument('--storage', default='fp64', choices=('fp64', 'fp32', 'fp16', 'bf16', 'bfp16'))
    ap.add_argument('--collision', default='MRT', choices=('MRT', 'SRT'))
    ap.add_argument('--size', type=int, default=256)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--mode', default='mlups', choices=('mlups', 'ttp'),
                    help='mlups: the throughput line; ttp: time to permeability, plain FP64 vs reduced storage')
    ap.add_argument('--storages', default='fp64,fp32,fp32+acc,bfp16+acc,fp32+warm0')
    ap.add_argument('--max-steps', type=int, default=400000)
    ap.add_argument('--io-write', type=int, default=500, help='io: VTI write interval')
    ap.add_argument('--io-restart', type=int, default=1000, help='io: checkpoint interval')
    ap.add_argument('--color-steps', type=int, default=50000, help='color-precision: steps of each run')
    ap.add_argument('--workload', default='scsp', choices=('scsp', 'color', 'color-precision', 'batch', 'operator',
                                                           'io'),
                    help='scsp: 256^3 single-phase cube; color: 128x128x256 two-phase color-gradient MRT; '
                         'batch: many uneven geometries in one launch; operator: the warm-start network '
                         '(forward + backward) on the tensor cores; io: output cost of a command-line run')
    ap.add_argument('--count', type=int, default=512, help='batch: number of geometries')
    ap.add_argument('--ttp-media', default='cube', choices=('cube', 'eval192'),
                    help='ttp: the 256^3 cube, or held-out 192^3 media')
    ap.add_argument('--seeds', type=int, default=8, help='ttp eval192: number of media')
    ap.add_argument('--media-index', default=None, help='ttp eval192: comma-separated media indices instead')
    ap.add_argument('--op-conv-only', action='store_true', help='operator: only the single-convolution roofline '
                                                                 '(3 warm-up + 20 timed launches)')
    ap.add_argument('--report', type=int, default=500, help='ttp: report interval in steps (the +acc '
                                                            'corrections act on report steps)')
    ap.add_argument('--block', type=int, default=2, help='ttp: block edge of the Darcy corrections (warm start, +acc)')
    ap.add_argument('--accel-at', default='500', help='ttp: report steps (step or step:block, comma separated) at '
                                                      'which +acc runs apply the block Darcy pressure correction')
    ap.add_argument('--accel-face', default='geometric', choices=('harmonic', 'geometric', 'arithmetic'))
    ap.add_argument('--accel-omega', type=float, default=1.0)
    ap.add_argument('--history', action='store_true', help='ttp: include (step, residual, K) of every report')
    ap.add_argument('--k-ref', type=float, default=None, help='ttp: reference (converged FP64) K for the band, '
                                                              'instead of running fp64')
    ap.add_argument('--warm-weights', default=str(Path(__file__).resolve().parent / 'lbflow_b200' / 'weights' /
                                                  'warmstart.pt'), help='ttp: trained warm-start operator')
    ap.add_argument('--check', type=int, default=8, help='batch: geometries re-solved alone in FP64')
    ap.add_argument('--ref-steps', type=int, default=3, help='reference arm: steps per reference process')
    ap.add_argument('--no-ttp', action='store_true', help='default line without the time-to-permeability runs')
    ap.add_argument('--no-others', action='store_true', help='default line without the other workloads\' rates')
    ap.add_argument('--cap16', type=int, default=0, help='ttp: step cap of 16-bit runs (0: --max-steps)')
    ap.add_argument('--ttp-runs', default='fp64,fp16+acc,fp16+mob',
                    help='runs of the default line\'s time-to-permeability object')
    ap.add_argument('--mob-weights', default=str(Path(__file__).resolve().parent / 'lbflow_b200' / 'weights' /
                                                 'mobility.pt'), help='trained block-mobility operator')
    ap.add_argument('--ref-procs', type=int, default=None, help='reference arm: cap on concurrent processes')
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == 'reference':
        return run_reference_arm(args)
    if args.mode == 'ttp':
        return time_to_permeability(args)
    if args.workload == 'color':
        return color_throughput(args)
    if args.workload == 'color-precision':
        return color_precision(args)
    if args.workload == 'batch':
        return batch_run(args)
    if args.workload == 'operator':
        return operator_run(args)
    if args.workload == 'io':
        return io_run(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120), device_id=torch.device('cuda', local))

    from lbflow_b200 import Engine
    geometry = make_geometry(args.size, 3.0, 0.22, seed=rank)
    N = geometry.size
    eng = Engine(geometry, LABELS, model='scsp', collision=args.collision, tau=(1.0,), rho=(1.0,),
                 storage=args.storage, device=local)
    nf = eng.fluid_nodes
    eng.initialize()
    eng.step(args.warmup)
    eng.synchronize()
    eng.check()

    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device('cuda', local))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t0.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            eng.step(1)
            ev[k][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total_ms = t0.elapsed_time(t1)
    launch_ms = statistics.fmean(a.elapsed_time(b) for a, b in ev)
    eng.check()
    if world > 1:
        tt = torch.tensor([total_ms], device='cuda')
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
        nn = torch.tensor([float(nf)], device='cuda', dtype=torch.float64)
        dist.all_reduce(nn)
        nf_all = float(nn.item())
    else:
        nf_all = float(nf)
    value = nf_all * args.steps / (total_ms / 1e3) / 1e6

    peak, peak_kind = measured_peaks()
    bytes_launch = nf * ALG_BYTES[args.storage]
    achieved = bytes_launch / (launch_ms / 1e3) / 1e9
    traffic = profile_traffic(args.storage)

    e2e = None
    if not args.no_e2e:
        eng.close()
        e2e = end_to_end(geometry, args, local)

    ttp = None
    if rank == 0 and world == 1 and not args.no_ttp and args.storage == 'fp64' and args.size % 8 == 0:
        ttp = ttp_line(args)
    others = None
    if rank == 0 and world == 1 and not args.no_others and args.storage == 'fp64':
        others = other_workloads(args, geometry)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, _ = reference_sample(steps=2, procs=1)

    if rank == 0:
        clk = clocks.summary()
        line = dict(metric=METRIC, value=value, unit='MLUPS', n_gpus=world, steps=args.steps,
                    warmup=args.warmup, ms_per_step=total_ms / args.steps, higher_is_better=True,
                    scaling='weak', vs_baseline=None, dtype=args.storage.replace('fp', 'f'),
                    data='synthetic',
                    config=dict(workload=f'D3Q19 {args.collision} single-phase porous cube {args.size}^3, '
                                         f'{args.storage} populations',
                                nx=args.size, ny=args.size, nz=args.size, porosity=0.22, sigma=3,
                                tau=1.0, g_x=1e-5, fluid_nodes=nf, total_voxels=N,
                                parallelism=f'replicas x{world}' if world > 1 else 'single GPU',
                                l2='inputs larger than L2 (populations %.2f GB)' % (2 * nf * 19 * ELEM[args.storage] / 1e9)),
                    roofline=dict(bound='hbm', achieved=achieved, peak=peak, unit='GB/s',
                                  frac=achieved / peak, traffic=traffic, peak_kind=peak_kind,
                                  bytes_per_launch=bytes_launch, launch_ms=launch_ms),
                    gpu_launches=args.steps,
                    clocks=clk, e2e=e2e, cpu_baseline=base, ttp=ttp, workloads=others)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def color_geometry():
    """Two-phase workload: 128 x 128 x 256 (x, y, z), sigma 2, porosity 0.30;
    pore voxels with z < 85 are phase A (label 75), the rest phase B (76)."""
    from lbflow_b200.geometry import porous_medium
    fluid = porous_medium((256, 128, 128), sigma=2.0, porosity=0.30, seed=0)
    g = np.where(fluid, 76, 255).astype(np.uint8)
    g[:85][fluid[:85]] = 75
    labels = {75: ('GV', 2e-6, 5, 0), 76: ('GV', 2e-6, 5, 1), 255: ('SD', 60.0, 0, 0)}
    return g, labels


def color_throughput(args):
    """Fluid MLUPS of the two-phase step (two launches per step) with its
    roofline: 2 * (2 * 19 * s) + 2 * 8 + 4 algorithmic bytes per fluid node."""
    import torch
    from lbflow_b200 import Engine
    torch.cuda.set_device(0)
    g, labels = color_geometry()
    storage = args.storage if args.storage in ('fp64', 'fp32', 'fp16', 'bf16') else 'fp64'
    eng = Engine(g, labels, model='color', collision=args.collision, tau=(1.0, 0.7), rho=(1.0, 1.0),
                 alpha0=1 / 3, sigma=1e-3, beta=0.7, storage=storage)
    nf = eng.fluid_nodes
    eng.initialize()
    eng.step(args.warmup)
    eng.synchronize()
    stream = torch.cuda.ExternalStream(eng.stream)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(args.steps // 4, 10)
    with ClockSampler(0) as clocks:
        t0.record(stream)
        eng.step(steps)
        t1.record(stream)
        torch.cuda.synchronize()
    eng.check()
    ms = t0.elapsed_time(t1)
    s = ELEM[storage]
    alg = 2 * (2 * 19 * s) + 2 * 8 + 4     # 16-bit: total + share, 2 bytes each per direction
    peak, kind = measured_peaks()
    achieved = nf * alg * steps / (ms / 1e3) / 1e9
    sums = eng.flux_sums()
    print(json.dumps(dict(metric='D3Q19 color-gradient MRT fluid MLUPS (128x128x256, porosity 0.30)',
                          value=nf * steps / (ms / 1e3) / 1e6, unit='MLUPS', steps=steps, ms_per_step=ms / steps,
                          dtype=storage, fluid_nodes=nf, gpu_launches=2 * steps,
                          roofline=dict(bound='hbm', achieved=achieved, peak=peak, frac=achieved / peak,
                                        unit='GB/s', bytes_per_node=alg, peak_kind=kind),
                          saturation_phase0=sums[8] / nf, clocks=clocks.summary())))
    eng.close()
    return 0


def color_precision(args):
    """The two-phase workload run to --color-steps (default 50,000) with FP64,
    FP32, FP16 and BF16 storage: phase-0 saturation, phase-0 mass drift over
    the run and the phase-fraction-weighted Darcy flux of each phase along the
    force (scripts/porous_media.py:20-44: means of phi_k u over all voxels),
    each storage's error against FP64, and the wall time."""
    import torch
    from lbflow_b200 import Engine
    torch.cuda.set_device(0)
    g, labels = color_geometry()
    N = g.size
    out = {}
    for storage in ('fp64', 'fp32', 'fp16', 'bf16'):
        with Engine(g, labels, model='color', collision=args.collision, tau=(1.0, 0.7), rho=(1.0, 1.0),
                    alpha0=1 / 3, sigma=1e-3, beta=0.7, storage=storage) as eng:
            eng.initialize()
            s0 = eng.flux_sums()
            eng.synchronize()
            t0 = time.perf_counter()
            eng.step(args.color_steps, macros=True)
            eng.synchronize()
            sec = time.perf_counter() - t0
            eng.check()
            s1 = eng.flux_sums()
            nf = eng.fluid_nodes
        out[storage] = dict(saturation_phase0=s1[8] / nf, mass_drift_phase0=(s1[6] - s0[6]) / s0[6],
                            mass_drift_phase1=(s1[7] - s0[7]) / s0[7],
                            darcy_flux_z=s1[2] / N, phase_flux_z=[s1[5] / N, (s1[2] - s1[5]) / N],
                            seconds=sec, mlups=nf * args.color_steps / sec / 1e6)
    ref = out['fp64']
    for k, v in out.items():
        v['saturation_rel_error'] = abs(v['saturation_phase0'] - ref['saturation_phase0']) / ref['saturation_phase0']
        v['darcy_flux_rel_error'] = abs(v['darcy_flux_z'] - ref['darcy_flux_z']) / abs(ref['darcy_flux_z'])
        v['phase_flux_rel_error'] = [abs(a - b) / abs(b) for a, b in zip(v['phase_flux_z'], ref['phase_flux_z'])]
    print(json.dumps(dict(metric='two-phase workload, reduced-precision storage against FP64',
                          workload='128x128x256 color-gradient MRT, sigma 2, porosity 0.30, inlet third phase A, '
                                   'tau 1/0.7, A 1e-3, beta 0.7, 60-degree walls, g_z 2e-6',
                          steps=args.color_steps, runs=out)))
    return 0


def io_run(args):
    """Output cost of a command-line run: the LBFlow binary on the 256^3 cube
    (FP64 MRT), once writing VTI fields every `--io-write` steps and a
    checkpoint every `--io-restart` steps, once writing only at the end; the
    timing line's field and checkpoint seconds per output and the wall-time
    overhead of the outputs."""
    import tempfile
    exe = ROOT / 'lbflow_b200' / 'lib' / 'LBFlow'
    geometry = make_geometry(args.size, 3.0, 0.22, seed=0)
    nz, ny, nx = geometry.shape
    steps, W, R = args.steps, args.io_write, args.io_restart

    def run(write, restart):
        with tempfile.TemporaryDirectory() as d:
            d = Path(d)
            geometry.tofile(d / 'geometry.raw')
            prm = (f'gridFile "geometry.raw";\ndimension {nz} {ny} {nx};\ndirections 19;\nfileType "uint8";\n'
                   f'latticeLen 1;\nstartTime 0;\nendTime {steps};\nwriteInterval {write};\n'
                   f'reportInterval {write};\nrestartInterval {restart};\nstopError 1e-12;\noutPath "field";\n'
                   f'logPath ".";\nreportDir 0;\nreportSlice 1 {nx - 2};\nfluidModel "scsp";\n'
                   f'equilModel "MRT";\nrexlationTime 1;\nlatticeSpeed 1;\nalpha0 0.33333333333333331;\n'
                   f'density 1;\ncontactAngle 90;\nsurfaceTension 0;\ninterfaceThickness 0.7;\n'
                   f'75 "GV" "1e-5" "1" "0"\n255 "SD" "90" "N/A" "N/A"\n')
            (d / 'input.prm').write_text(prm)
            t0 = time.perf_counter()
            r = subprocess.run([str(exe), 'input.prm'], cwd=d, capture_output=True, text=True)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError('LBFlow failed: ' + r.stdout[-500:])
            t = [json.loads(l[len('LBFlowTiming '):]) for l in r.stdout.splitlines()
                 if l.startswith('LBFlowTiming ')][0]
            files = sorted(p.name for p in d.iterdir() if p.name.startswith('field'))
            size = sum((d / f).stat().st_size for f in files)
            return t, wall, files, size

    quiet, wq, _, _ = run(steps, steps * 10)
    loud, wl, files, size = run(W, R)
    n_vti = steps // W + 1
    n_rst = steps // R
    print(json.dumps(dict(
        metric='command-line output cost, 256^3 FP64 MRT', unit='s',
        value=(loud['run_seconds_max'] - quiet['run_seconds_max']) / (n_vti - 2 + n_rst),
        higher_is_better=False, steps=steps, write_interval=W, restart_interval=R,
        vti_files=n_vti, checkpoints=n_rst, bytes_written=size,
        seconds_per_vti=loud['fields_diagnostics_seconds_max'] / n_vti,
        seconds_per_checkpoint=loud['checkpoint_seconds_max'] / max(n_rst, 1),
        run_seconds_with_outputs=loud['run_seconds_max'], run_seconds_final_only=quiet['run_seconds_max'],
        numerical_seconds=[loud['numerical_seconds_max'], quiet['numerical_seconds_max']],
        process_wall_seconds=[wl, wq])))
    return 0


def _batch_member(spec):
    from lbflow_b200.geometry import porous_medium
    shape, sigma, poro, seed = spec
    return np.where(porous_medium(shape, sigma=sigma, porosity=poro, seed=seed), 75, 255).astype(np.uint8)


def batch_geometries(count, seed=2024):
    """Batched workload: per geometry, edges drawn from {32,48,64,96,128} per
    axis, sigma ~ U[1.5, 6], porosity ~ U[0.10, 0.35], tau ~ U[0.6, 1.4]."""
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    specs, taus = [], []
    for k in range(count):
        shape = tuple(int(v) for v in rng.choice([32, 48, 64, 96, 128], size=3))
        specs.append((shape, float(rng.uniform(1.5, 6.0)), float(rng.uniform(0.10, 0.35)), seed * 1000 + k))
        taus.append(float(rng.uniform(0.6, 1.4)))
    with mp.get_context('spawn').Pool(min(16, os.cpu_count() or 1)) as pool:
        geoms = pool.map(_batch_member, specs, chunksize=4)
    return geoms, taus, specs


def batch_run(args):
    """All geometries in one batch, each converged to the 1e-6 criterion and
    retired; aggregate fluid MLUPS; permeability of a sample re-solved alone
    with the plain FP64 engine.  Under torchrun the geometries are split over
    the ranks (one GPU each, batch.converge_sharded): no data-path
    collective, the per-geometry results gathered host-side over gloo, the
    time the slowest rank's."""
    import torch
    from lbflow_b200 import Engine
    from lbflow_b200.batch import Batch, converge_sharded
    from lbflow_b200.permeability import converge
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group('gloo', timeout=timedelta(seconds=600))
    t0 = time.perf_counter()
    geoms, taus, specs = batch_geometries(args.count)
    gen_s = time.perf_counter() - t0
    storage = args.storage if args.storage in ('fp64', 'fp32', 'fp16') else 'fp64'
    tune = None
    if world > 1:
        dist.barrier()
        res = converge_sharded(geoms, taus, LABELS, 1e-5, rank=rank, world=world, device=local,
                               collision=args.collision, storage=storage, report=1000, tol=1e-6,
                               max_steps=args.max_steps)
        nodes = res['nodes']
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return 0
    else:
        b = Batch(geoms, taus, LABELS, collision=args.collision, storage=storage)
        b.initialize()
        tune = b.autotune(steps=6)
        res = b.converge(1e-5, report=1000, tol=1e-6, max_steps=args.max_steps)
        nodes = b.fluid_nodes()
        b.close()
    check = []
    for k in range(min(args.check, args.count)):
        e = Engine(geoms[k], LABELS, collision=args.collision, tau=(taus[k],))
        r = converge(e, taus[k], 1e-5, report=1000, tol=1e-6, max_steps=args.max_steps)
        e.close()
        check.append(dict(geometry=k, shape=list(specs[k][0]), K_batch=float(res['K'][k]), K_fp64=r['K'],
                          rel_error=abs(res['K'][k] - r['K']) / abs(r['K']), steps=int(res['steps'][k])))
    print(json.dumps(dict(metric='batched D3Q19 MRT aggregate fluid MLUPS',
                          value=res['mlups'], unit='MLUPS', n_gpus=world,
                          scaling='strong' if world > 1 else None, geometries=args.count, fluid_nodes=nodes,
                          converged=int(res['converged'].sum()), seconds=res['seconds'],
                          steps_max=int(res['steps'].max()), dtype=storage, autotune=tune,
                          generation_seconds=gen_s, permeability_check=check,
                          max_rel_error=max((c['rel_error'] for c in check), default=None))))
    return 0


def ttp_media(args):
    """Media of the time-to-permeability runs: the 256^3 cube of the MLUPS line
    (sigma 3, porosity 0.22), or --ttp-media eval192: 192^3 media with
    sigma ~ U[2, 5] and porosity ~ U[0.15, 0.30] from seeds that no training
    medium uses."""
    if args.ttp_media == 'cube':
        return [dict(name=f'cube{args.size}', geometry=make_geometry(args.size, 3.0, 0.22, seed=0),
                     sigma=3.0, porosity=0.22, seed=0)]
    out = []
    pick = [int(v) for v in args.media_index.split(',')] if args.media_index else range(args.seeds)
    for k in pick:
        seed = 900000 + k
        rng = np.random.default_rng([seed, 5])
        sigma, por = float(rng.uniform(2.0, 5.0)), float(rng.uniform(0.15, 0.30))
        out.append(dict(name=f'eval192_{k}', geometry=make_geometry(192, sigma, por, seed=seed), sigma=sigma,
                        porosity=por, seed=seed))
    return out


def ttp_medium(med, args, net, storages):
    """Time-to-permeability runs of one medium; returns (runs, histories)."""
    import torch
    from lbflow_b200 import Engine
    from lbflow_b200 import warmstart as ws
    from lbflow_b200.permeability import converge
    geometry = med['geometry']
    fluid = torch.from_numpy(geometry != 255).cuda()
    names = storages.split(',')
    # One-time set-up outside the timed runs, as CUDA context creation is:
    # CUDA kernels (the library's and torch's size-dependent variants) load
    # on first launch, so a throwaway engine of each storage takes one step,
    # one block correction and, for warm starts, one network inference on
    # this medium.  No state carries over into the timed runs.
    for storage in sorted({n.split('+')[0] for n in names}):
        with Engine(geometry, LABELS, model='scsp', collision=args.collision, tau=(1.0,), rho=(1.0,),
                    storage=storage) as e:
            e.initialize()
            e.step(1, macros=True)
            if any('+acc' in n for n in names):
                ws.DarcyAccelerator(e, fluid, 1e-5, block=args.block, at=(1,))(1)
            if net is not None:
                ws.predict(net, fluid, 1.0, 1e-5)
            if any('+mob' in n for n in names):
                ws.mobility_start(e, args.mob_net, fluid, 1.0, 1e-5, block=args.block)
            e.check()
    torch.cuda.synchronize()
    runs, hist = {}, {}
    for name in names:
        storage, *mods = name.split('+')
        start = acc = None
        eng = Engine(geometry, LABELS, model='scsp', collision=args.collision, tau=(1.0,), rho=(1.0,),
                     storage=storage)
        for mod in mods:
            kind = mod.rstrip('0123456789')
            block = int(mod[len(kind):]) if mod[len(kind):] else args.block
            if kind in ('warm', 'warmv', 'flux', 'rho'):
                mode = {'warm': 'darcy', 'warmv': 'darcy', 'flux': 'flux', 'rho': 'none'}[kind] if block else 'none'
                start = (lambda b=block, m=mode, v=(kind == 'warmv'):
                         ws.warm_start(eng, net, fluid, 1.0, 1e-5, block=b, mode=m, velocity=v))
            elif kind == 'mob':
                start = (lambda b=block: ws.mobility_start(eng, args.mob_net, fluid, 1.0, 1e-5, block=b))
            elif kind == 'acc':
                sched = [tuple(int(v) for v in item.split(':')) if ':' in item else int(item)
                         for item in args.accel_at.split(',')]
                acc = ws.DarcyAccelerator(eng, fluid, 1e-5, block=block, at=sched, face=args.accel_face,
                                          omega=args.accel_omega)
        # 16-bit storage: stochastic rounding keeps the velocity residual
        # near 1e-4, above LBFlow's 1e-6, so such runs end at their step cap
        # and their stall watch sits above that noise.
        sixteen = storage in ('fp16', 'bf16', 'bfp16')
        cap = min(args.max_steps, args.cap16) if sixteen and args.cap16 else args.max_steps
        r = converge(eng, 1.0, 1e-5, report=args.report, tol=1e-6, max_steps=cap, warm=start,
                     accelerate=acc, stall_floor=1e-2 if sixteen else None)
        hist[name] = r['history']
        runs[name] = dict(steps=r['steps'], seconds=r['seconds'], K=r['K'], converged=r['converged'],
                          fallback=r['fallback'], fluid_nodes=eng.fluid_nodes,
                          mlups=eng.fluid_nodes * r['steps'] / r['seconds'] / 1e6)
        if acc is not None:
            runs[name]['accelerator'] = dict(applied=acc.applied, seconds=acc.seconds,
                                             cg_iterations=acc.iterations, phases=acc.phases)
        if args.history:
            runs[name]['history'] = [(h[0], h[1], h[3]) for h in r['history']]
        eng.close()
    return runs, hist


def band_summary(runs, hist, k_ref):
    """Adds K error, steps/seconds to the 1e-3 band and speed-ups against fp64."""
    from lbflow_b200.permeability import time_to_band
    base = runs.get('fp64')
    for k, v in runs.items():
        if k_ref:
            v['K_rel_error_vs_fp64'] = abs(v['K'] - k_ref) / abs(k_ref)
            band = time_to_band(hist[k], k_ref, 1e-3)
            v['to_1e-3_band'] = dict(steps=band[0], seconds=band[1]) if band else None
        if base:
            v['speedup_vs_fp64'] = base['seconds'] / v['seconds']
    if base and base.get('to_1e-3_band'):
        b0 = base['to_1e-3_band']['seconds']
        for k, v in runs.items():
            if v.get('to_1e-3_band'):
                v['to_1e-3_band']['speedup_vs_fp64'] = b0 / v['to_1e-3_band']['seconds']


def load_networks(args, storages):
    from lbflow_b200 import warmstart as ws
    net = None
    if any(m in r for r in storages.split(',') for m in ('+warm', '+flux', '+rho')):
        net, _ = ws.load(args.warm_weights)
    args.mob_net = None
    if '+mob' in storages:
        args.mob_net, _ = ws.load_mobility(args.mob_weights)
    return net


def time_to_permeability(args):
    """Wall time to LBFlow's convergence criterion (report every --report
    steps, relative velocity change < 1e-6 three times in a row) and to K within 1e-3
    of the plain FP64 result, for each run of --storages: a storage name
    (fp64, fp32, fp16, bf16, bfp16) starts from rest as LBFlow does; a
    '+warm' suffix starts from the learned warm start (feature computation,
    network inference and the block-scale Darcy pressure with --block voxel
    blocks, inside the timed region); '+warmB' sets the block edge B (0: the
    network's fields only); '+fluxB' uses the flux-divergence correction
    instead; warm starts set the predicted density only ('+warmvB' also the
    predicted velocity); '+mobB' starts from the block Darcy pressure of the
    learned block mobilities (warmstart.mobility_start); '+accB' applies the
    in-run block Darcy correction (warmstart.DarcyAccelerator) at the
    --accel-at report steps.  K = nu <u_x> / g."""
    import torch
    torch.cuda.set_device(0)
    net = load_networks(args, args.storages)
    media = ttp_media(args)
    results = []
    for med in media:
        runs, hist = ttp_medium(med, args, net, args.storages)
        base = runs.get('fp64')
        kref = args.k_ref if args.k_ref else (base['K'] if base else None)
        band_summary(runs, hist, kref)
        results.append(dict(medium=med['name'], sigma=med['sigma'], porosity=med['porosity'], seed=med['seed'],
                            runs=runs))
        print(json.dumps(results[-1]), flush=True)
    summary = {}
    for name in args.storages.split(','):
        sp = [r['runs'][name]['to_1e-3_band']['speedup_vs_fp64'] for r in results
              if r['runs'][name].get('to_1e-3_band') and 'speedup_vs_fp64' in r['runs'][name]['to_1e-3_band']]
        ke = [r['runs'][name].get('K_rel_error_vs_fp64') for r in results if 'K_rel_error_vs_fp64' in r['runs'][name]]
        st = [r['runs'][name]['to_1e-3_band']['steps'] for r in results if r['runs'][name].get('to_1e-3_band')]
        summary[name] = dict(band_speedup_median=float(np.median(sp)) if sp else None,
                             band_speedup_min=float(min(sp)) if sp else None,
                             band_steps_median=float(np.median(st)) if st else None,
                             K_rel_error_max=float(max(ke)) if ke else None,
                             fallbacks=sum(bool(r['runs'][name]['fallback']) for r in results))
    print(json.dumps(dict(metric='time to permeability (K within 1e-3 of converged FP64; 1e-6 convergence)',
                          media=args.ttp_media, report_interval=args.report,
                          workload=f'D3Q19 {args.collision}, tau 1, g_x 1e-5, periodic porous media',
                          summary=summary)))
    return 0


def _timed_steps(stream, run, steps):
    """CUDA-event milliseconds of run() (which enqueues `steps` steps) on `stream`."""
    import torch
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    run()
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1)


def other_workloads(args, geometry):
    """Sub-objects of the default line for the other workloads, each device-
    timed with CUDA events after warm-up steps: the 256^3 cube with FP32 and
    FP16 storage, the two-phase 128x128x256 medium (FP64 and FP16 storage)
    and 64 uneven media in one batched launch (FP64)."""
    import torch
    from lbflow_b200 import Engine
    from lbflow_b200.batch import Batch
    peak, kind = measured_peaks()
    out = {}
    for storage in ('fp32', 'fp16'):
        with Engine(geometry, LABELS, model='scsp', collision=args.collision, tau=(1.0,), rho=(1.0,),
                    storage=storage) as e:
            e.initialize()
            e.step(args.warmup)
            steps = 40
            ms = _timed_steps(torch.cuda.ExternalStream(e.stream), lambda: e.step(steps), steps)
            e.check()
            nf = e.fluid_nodes
        b = ALG_BYTES[storage]
        out[f'scsp_{storage}'] = dict(value=nf * steps / (ms / 1e3) / 1e6, unit='MLUPS', ms_per_step=ms / steps,
                                      bytes_per_node=b, frac=nf * b * steps / (ms / 1e3) / 1e9 / peak)
    g, labels = color_geometry()
    for storage in ('fp64', 'fp16'):
        with Engine(g, labels, model='color', collision=args.collision, tau=(1.0, 0.7), rho=(1.0, 1.0),
                    alpha0=1 / 3, sigma=1e-3, beta=0.7, storage=storage) as e:
            e.initialize()
            e.step(args.warmup)
            steps = 40
            ms = _timed_steps(torch.cuda.ExternalStream(e.stream), lambda: e.step(steps), steps)
            e.check()
            nf = e.fluid_nodes
        b = 2 * (2 * 19 * ELEM[storage]) + 2 * 8 + 4
        out[f'color_{storage}'] = dict(value=nf * steps / (ms / 1e3) / 1e6, unit='MLUPS', ms_per_step=ms / steps,
                                       bytes_per_node=b, frac=nf * b * steps / (ms / 1e3) / 1e9 / peak,
                                       workload='128x128x256 two-phase color MRT, sigma 2, porosity 0.30')
    geoms, taus, _ = batch_geometries(64)
    with Batch(geoms, taus, LABELS, collision=args.collision, storage='fp64') as bt:
        bt.initialize()
        tune = bt.autotune(steps=6)
        bt.step(64)
        steps = 640
        ms = _timed_steps(torch.cuda.ExternalStream(bt.stream), lambda: bt.step(steps), steps)
        bt.check()
        nf = bt.fluid_nodes()
    out['batch_fp64'] = dict(value=nf * steps / (ms / 1e3) / 1e6, unit='MLUPS', ms_per_step=ms / steps,
                             bytes_per_node=308, frac=nf * 308 * steps / (ms / 1e3) / 1e9 / peak,
                             workload='64 uneven media (edges 32-128, porosity 0.10-0.35) in one launch',
                             fluid_nodes=int(nf), autotune=tune)
    out['peak_gbs'] = peak
    out['peak_kind'] = kind
    return out


def ttp_line(args):
    """The time-to-permeability sub-object of the default line: the 256^3
    cube of the throughput workload, FP64 from rest (LBFlow's method; its
    converged K is the reference) against the chosen forms."""
    net = load_networks(args, args.ttp_runs)
    med = ttp_media(argparse.Namespace(ttp_media='cube', size=args.size))[0]
    if not args.cap16:
        args.cap16 = 40000
    runs, hist = ttp_medium(med, args, net, args.ttp_runs)
    k_ref = runs['fp64']['K'] if runs.get('fp64', {}).get('converged') else None
    band_summary(runs, hist, k_ref)
    slim = {}
    for name, v in runs.items():
        b = v.get('to_1e-3_band') or {}
        slim[name] = dict(steps_to_band=b.get('steps'), seconds_to_band=b.get('seconds'),
                          band_speedup_vs_fp64=b.get('speedup_vs_fp64'), converged=v['converged'],
                          steps_to_converge=v['steps'], seconds_to_converge=v['seconds'], K=v['K'],
                          K_rel_error_vs_fp64=v.get('K_rel_error_vs_fp64'), fallback=v['fallback'])
        if 'accelerator' in v:
            slim[name]['correction_seconds'] = v['accelerator']['seconds']
    return dict(metric='time to permeability within 1e-3 of the converged FP64 K (wall seconds)',
                medium=f'{args.size}^3 cube, sigma 3, porosity 0.22, seed 0', report_interval=args.report,
                convergence='LBFlow criterion: relative velocity change < 1e-6 at 3 consecutive reports; '
                            f'16-bit runs (rounding noise above that criterion) end at {args.cap16} steps',
                K_ref=k_ref, runs=slim,
                notes='fp64: the plain path from rest (LBFlow); +acc: one block Darcy pressure correction at '
                      'step 500 from the run\'s own block mobilities; +mob: learned start -- the block '
                      'mobility network, the block Darcy pressure at t = 0, velocity at rest')


def operator_run(args):
    """Training step of the warm-start operator: forward + backward of the
    4-level U-Net on a batch of 2 x 96^3 media, every convolution on the
    tcgen05 kernels.  value = model TFLOP/s (3 x forward FLOPs per step).
    The roofline line is for the heaviest single convolution launch (the
    64-channel 3x3x3 periodic convolution at 2 x 48^3, forward), timed per
    launch with CUDA events and compared with the measured bf16 peak."""
    import torch
    from lbflow_b200 import conv
    from lbflow_b200 import warmstart as ws
    torch.cuda.set_device(0)
    d = json.loads((ROOT / 'MEASURED_PEAKS.json').read_text()) if (ROOT / 'MEASURED_PEAKS.json').exists() else {}
    peak = float(d.get('bf16_tflops', 1590.0))
    net = ws.WarmStartNet(seed=0).cuda()
    rng = np.random.default_rng(0)
    fl = torch.from_numpy(rng.random((2, 96, 96, 96)) < 0.3).cuda()
    x = ws.features(fl)
    R = torch.randn(2, 96, 96, 96, 8, device='cuda').to(torch.bfloat16)
    flops = 3 * net.flops(96 ** 3) * 2

    def step():
        net.zero_grad(set_to_none=True)
        y = net(x)
        (y.float() * R.float()).sum().backward()

    steps = max(5, min(args.steps, 50))
    ms = float('nan')
    clocks = None
    if not args.op_conv_only:
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            t0.record()
            for _ in range(steps):
                step()
            t1.record()
            torch.cuda.synchronize()
        clocks = clk.summary()
        conv.check()
        ms = t0.elapsed_time(t1) / steps
    # Heaviest single launch: 64 -> 64 channel 3x3x3 conv at 2 x 48^3 (level 3 of a 192^3 input).
    xa = torch.randn(2, 48, 48, 48, 64, device='cuda').to(torch.bfloat16)
    w = torch.randn(64, 64, 3, 3, 3, device='cuda') * 0.05
    b = torch.zeros(64, device='cuda')
    lf = 2 * 2 * 48 ** 3 * 27 * 64 * 64
    for _ in range(3):
        conv.conv3(xa, w, b, 0.1)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
    for a, c in ev:
        a.record()
        conv.conv3(xa, w, b, 0.1)
        c.record()
    torch.cuda.synchronize()
    conv.check()
    launch_ms = statistics.fmean(a.elapsed_time(c) for a, c in ev)
    achieved = lf / (launch_ms / 1e3) / 1e12
    print(json.dumps(dict(metric='warm-start operator training step, model TFLOP/s', value=flops / (ms / 1e3) / 1e12,
                          unit='TFLOP/s', steps=steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True,
                          dtype='bf16 (fp32 accumulate)', data='synthetic',
                          config=dict(workload='4-level U-Net, 2 x 96^3 media, forward + backward',
                                      params=sum(p.numel() for p in net.parameters()), flops_per_step=flops),
                          roofline=dict(bound='tensor', achieved=achieved, peak=peak, unit='TFLOP/s',
                                        frac=achieved / peak, traffic=None, peak_kind='measured burst bf16',
                                        kernel='igemm conv3 64->64 at 2x48^3 (forward)', launch_ms=launch_ms),
                          gpu_launches=None, clocks=clocks)))
    return 0

def end_to_end(geometry, args, device, repeats=5):
    """Same metric through the C ABI with host buffers: the uint8 geometry
    from the host (classified on the device), initialization, K steps each
    followed by the read-back of the step's flux and mass sums (the numbers
    K is computed from), then the final density and velocity fields in the
    VTI layout into page-locked host memory.  The page-locked output buffer
    is allocated before the timed region, as a caller reusing it would.
    Repeated `repeats` times with a fresh engine each; the median run is
    reported, with the seconds of its phases."""
    from lbflow_b200 import Engine, HostBuffer
    import torch
    fields = HostBuffer(4 * geometry.size)
    fields.array[::512] = 0.0          # touch the pages before timing
    # The step's input (the voxel labels) in page-locked memory, as the
    # caller of a production run holds it.
    gbuf = HostBuffer(geometry.size, dtype=np.uint8)
    geom = gbuf.array.reshape(geometry.shape)
    geom[...] = geometry
    runs = []
    for _ in range(repeats):
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng = Engine(geom, LABELS, model='scsp', collision=args.collision, tau=(1.0,), rho=(1.0,),
                     storage=args.storage, device=device)
        t1 = time.perf_counter()
        eng.initialize()
        sums = None
        for _ in range(args.steps):
            eng.step(1, macros=True)
            sums = eng.flux_sums()
        t2 = time.perf_counter()
        eng.fields_dense_async(fields.ptr.value, fields.count)
        eng.synchronize()
        eng.check()
        t3 = time.perf_counter()
        nf = eng.fluid_nodes
        eng.close()
        ok = bool(np.isfinite(fields.array[::4097]).all()) and sums is not None and np.isfinite(sums).all()
        if not ok:
            raise RuntimeError('end-to-end run produced non-finite output')
        runs.append(dict(seconds=t3 - t, create=t1 - t, steps=t2 - t1, fields=t3 - t2))
    fields.close()
    del geom
    gbuf.close()
    runs.sort(key=lambda r: r['seconds'])
    med = runs[len(runs) // 2]
    h2d = geometry.nbytes + 256 * 24
    d2h = 9 * 8 * args.steps + 4 * 8 * geometry.size
    return dict(value=nf * args.steps / med['seconds'] / 1e6, unit='MLUPS',
                h2d_bytes_per_step=h2d / args.steps, d2h_bytes_per_step=d2h / args.steps,
                seconds=med['seconds'], phases={k: med[k] for k in ('create', 'steps', 'fields')},
                repeats=repeats, seconds_all=[r['seconds'] for r in runs])


if __name__ == '__main__':
    sys.exit(main())
