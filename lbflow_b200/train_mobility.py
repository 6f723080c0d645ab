"""Train the block-mobility operator of the learned start (warmstart.MobilityNet).

    python -m lbflow_b200.train_mobility --count 2000 --out lbflow_b200/weights/mobility.pt

Data: seeded porous media from the Gaussian-filtered-noise recipe with edges
drawn per axis from {64, 96, 128}, sigma ~ U[1.5, 6], porosity ~ U[0.12, 0.35]
(train_warmstart.draw; media that do not percolate along x are redrawn),
tau = 1, force g = 1e-5 along +x, MRT collision.  The batched engine runs
every medium warmstart.MOB_STEPS steps from rest; the block mobilities the
Darcy correction would estimate from that state (warmstart.block_mobility)
are the targets.  5% of the media (seed % 20 == 0) are held out and
reported.  Geometries are drawn in a spawn-started process pool before the
first GPU call.
"""
import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np

from .train_warmstart import EDGES, LABELS, draw

G = 1e-5
TAU = 1.0


def run_chunk(items, log):
    """Batched run of MOB_STEPS steps from rest; returns per-medium
    (fluid, target, weight) on the GPU and the meta records."""
    import torch
    from .batch import Batch
    from . import warmstart as ws
    geoms = [np.where(f, 75, 255).astype(np.uint8) for f, _, _ in items]
    out = []
    t0 = time.perf_counter()
    with Batch(geoms, [TAU] * len(geoms), LABELS, collision='MRT', storage='fp64') as b:
        b.initialize()
        b.step(ws.MOB_STEPS, macros=True)
        b.check()
        for k, (f, _, meta) in enumerate(items):
            r, u = b.macros(k)
            fl = torch.from_numpy(f).cuda()
            t, w = ws.mobility_targets(torch.from_numpy(r).cuda(), torch.from_numpy(u).cuda(), fl, TAU, G)
            out.append((fl, t, w, dict(meta, tau=TAU)))
    log(f'  chunk of {len(items)} media: {ws.MOB_STEPS} steps + targets in {time.perf_counter() - t0:.1f}s')
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--count', type=int, default=2000)
    ap.add_argument('--seed0', type=int, default=300000)
    ap.add_argument('--chunk', type=int, default=250)
    ap.add_argument('--iters', type=int, default=4000)
    ap.add_argument('--lr', type=float, default=2e-3)
    ap.add_argument('--batch-voxels', type=int, default=2 * 96 ** 3)
    ap.add_argument('--out', default='lbflow_b200/weights/mobility.pt')
    ap.add_argument('--log', default=None)
    args = ap.parse_args(argv)
    lines = []

    def log(s):
        print(s, flush=True)
        lines.append(s)

    t_start = time.perf_counter()
    seeds = list(range(args.seed0, args.seed0 + args.count))
    with mp.get_context('spawn').Pool(max(1, min(32, (os.cpu_count() or 2) - 1))) as pool:
        media = pool.map(draw, seeds, chunksize=4)
    t_gen = time.perf_counter() - t_start
    log(f'generated {len(media)} media in {t_gen:.1f}s (edges {EDGES})')

    import torch
    from . import warmstart as ws
    media.sort(key=lambda m: (m[2]['shape'], m[2]['seed']))
    samples = []
    t0 = time.perf_counter()
    for i in range(0, len(media), args.chunk):
        samples += run_chunk(media[i:i + args.chunk], log)
    t_data = time.perf_counter() - t0
    held = [s for s in samples if s[3]['seed'] % 20 == 0]
    train = [s for s in samples if s[3]['seed'] % 20 != 0]
    net = ws.MobilityNet(seed=0).cuda()
    t0 = time.perf_counter()
    hist = ws.train_mobility(net, [s[:3] for s in train], iters=args.iters, lr=args.lr,
                             batch_voxels=args.batch_voxels, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ev_train = ws.evaluate_mobility(net, [s[:3] for s in train[:64]], TAU)
    ev_held = ws.evaluate_mobility(net, [s[:3] for s in held], TAU)

    def summary(ev):
        a = lambda k: float(np.median([e[k] for e in ev])) if ev else float('nan')
        return dict(n=len(ev), log_mob_rms_median=a('log_mob_rms'), log_mob_corr_median=a('log_mob_corr'))

    meta = dict(count=len(samples), train=len(train), held_out=len(held), tau=TAU, g=G, steps=ws.MOB_STEPS,
                block=ws.MOB_BLOCK, iters=args.iters, lr=args.lr, batch_voxels=args.batch_voxels,
                norm=net.norm.tolist(), seconds=dict(generate=t_gen, data=t_data, train=t_train),
                loss_history=hist, train_eval=summary(ev_train), held_out_eval=summary(ev_held),
                held_out_media=[dict(e, **m) for e, (_, _, _, m) in zip(ev_held, held)])
    log(json.dumps({k: meta[k] for k in ('train_eval', 'held_out_eval', 'seconds', 'norm')}))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    ws.save_mobility(net, args.out, meta)
    if args.log:
        with open(args.log, 'w') as fh:
            json.dump(dict(meta, log=lines), fh, indent=1)
    return 0


if __name__ == '__main__':
    raise SystemExit(main())
