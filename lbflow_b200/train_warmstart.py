"""Train the warm-start operator on steady fields from the batched solver.

    python -m lbflow_b200.train_warmstart --count 2000 --out lbflow_b200/weights/warmstart.pt

Data: seeded porous media from the Gaussian-filtered-noise recipe with edges
drawn per axis from {64, 96, 128}, sigma ~ U[1.5, 6], porosity ~ U[0.12, 0.35]
and tau ~ U[0.6, 1.4], force g = 1e-5 along +x, MRT collision, run with the
batched engine (lbf_batch_*) until LBFlow's residual criterion holds at
--tol.  The steady (u, rho) of each medium becomes the geometry-only target
(k = u nu / g, pi = (rho - rho0) / 3g) of warmstart.targets.  5% of the media
are held out and reported.  Geometries are drawn in a spawn-started process
pool before the first GPU call.
"""
import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np

LABELS = {75: ('GV', 1e-5, 1, 0), 255: ('SD', 90.0, 0, 0)}
G = 1e-5
EDGES = (64, 96, 128)


def draw(seed):
    """One training medium: (fluid mask, tau, description).  Media whose pore
    space does not cross the box along x (no flux under the force) are
    redrawn from the next sub-seed."""
    from lbflow_b200.geometry import percolates, porous_medium
    for attempt in range(50):
        rng = np.random.default_rng([seed, 2027, attempt])
        shape = tuple(int(v) for v in rng.choice(EDGES, size=3))
        sigma = float(rng.uniform(1.5, 6.0))
        por = float(rng.uniform(0.12, 0.35))
        tau = float(rng.uniform(0.6, 1.4))
        fluid = porous_medium(shape, sigma, por, seed=seed * 64 + attempt)
        if percolates(fluid, axis=-1):
            break
    return fluid, tau, dict(seed=seed, attempt=attempt, shape=shape, sigma=sigma, porosity=por, tau=tau)


def solve(items, storage, tol, max_steps, log):
    """Converge a chunk of media together; returns per-medium (mask, target) on the GPU."""
    import torch
    from lbflow_b200.batch import Batch
    from lbflow_b200.warmstart import targets
    geoms = [np.where(f, 75, 255).astype(np.uint8) for f, _, _ in items]
    out = []
    with Batch(geoms, [t for _, t, _ in items], LABELS, collision='MRT', storage=storage) as b:
        t0 = time.perf_counter()
        res = b.converge(G, report=1000, tol=tol, max_steps=max_steps)
        log(f'  chunk of {len(items)}: {res["updates"] / 1e9:.1f}e9 updates in {res["seconds"]:.1f}s '
            f'({res["mlups"]:.0f} MLUPS), converged {int(res["converged"].sum())}, '
            f'steps max {int(res["steps"].max())}')
        for k, (f, tau, meta) in enumerate(items):
            r, u = b.macros(k)
            meta = dict(meta, steps=int(res['steps'][k]), K=float(res['K'][k]),
                        converged=bool(res['converged'][k]))
            out.append((torch.from_numpy(f).cuda(), torch.from_numpy(targets(r, u, tau, G)).cuda(), meta))
        log(f'  solved + copied in {time.perf_counter() - t0:.1f}s')
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--count', type=int, default=2000)
    ap.add_argument('--seed0', type=int, default=100000)
    ap.add_argument('--chunk', type=int, default=250)
    ap.add_argument('--storage', default='fp64')
    ap.add_argument('--tol', type=float, default=1e-5)
    ap.add_argument('--max-steps', type=int, default=60000)
    ap.add_argument('--iters', type=int, default=3000)
    ap.add_argument('--lr', type=float, default=2e-3)
    ap.add_argument('--batch-voxels', type=int, default=2 * 96 ** 3)
    ap.add_argument('--out', default='lbflow_b200/weights/warmstart.pt')
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
    log(f'generated {len(media)} media in {t_gen:.1f}s')

    import torch
    from lbflow_b200 import warmstart as ws

    samples = []
    t0 = time.perf_counter()
    # Group media of one shape together so that chunks have similar run lengths.
    media.sort(key=lambda m: (m[2]['shape'], m[2]['seed']))
    for i in range(0, len(media), args.chunk):
        samples += solve(media[i:i + args.chunk], args.storage, args.tol, args.max_steps, log)
    t_solve = time.perf_counter() - t0
    log(f'solved {len(samples)} media in {t_solve:.1f}s')

    # Media that did not reach --tol within --max-steps are reported, not learned from.
    good = [s for s in samples if s[2]['converged']]
    held = [s for s in good if s[2]['seed'] % 20 == 0]
    train = [s for s in good if s[2]['seed'] % 20 != 0]
    net = ws.WarmStartNet(seed=0).cuda()
    t0 = time.perf_counter()
    hist = ws.train(net, [(f, t) for f, t, _ in train], iters=args.iters, lr=args.lr,
                    batch_voxels=args.batch_voxels, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    log(f'trained {args.iters} iterations in {t_train:.1f}s')
    ev_train = ws.evaluate(net, [(f, t) for f, t, _ in train[:64]])
    ev_held = ws.evaluate(net, [(f, t) for f, t, _ in held])

    def summary(ev):
        a = lambda k: float(np.median([e[k] for e in ev])) if ev else float('nan')
        return dict(n=len(ev), k_rel_l2_median=a('k_rel_l2'), pi_rel_l2_median=a('pi_rel_l2'),
                    K_rel_err_median=a('K_rel_err'))

    meta = dict(count=len(samples), train=len(train), held_out=len(held), tol=args.tol, storage=args.storage,
                iters=args.iters, lr=args.lr, batch_voxels=args.batch_voxels,
                seconds=dict(generate=t_gen, solve=t_solve, train=t_train),
                loss_history=hist, train_eval=summary(ev_train), held_out_eval=summary(ev_held),
                held_out_media=[dict(e, **m) for e, (_, _, m) in zip(ev_held, held)],
                scale=net.scale.tolist(), not_converged=int(sum(not m['converged'] for _, _, m in samples)))
    log(json.dumps({k: meta[k] for k in ('train_eval', 'held_out_eval', 'seconds', 'not_converged')}))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    ws.save(net, args.out, meta)
    if args.log:
        with open(args.log, 'w') as fh:
            json.dump(dict(meta, log=lines), fh, indent=1)
    return 0


if __name__ == '__main__':
    raise SystemExit(main())
