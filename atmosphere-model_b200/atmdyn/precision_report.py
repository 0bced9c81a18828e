"""Error of the mixed-precision form against the FP64 form.

    python -m atmdyn.precision_report [--n 2048] [--nlay 64] [--steps 50,100,200] [--seed 1]

Runs the seeded jet case (the precision-form workload: 2048 x 2048 x 64,
dt = 30 s, remap every 8 steps, seed 1) in the FP64 form and in the mixed
form side by side on one GPU, and prints one JSON object with, at each
requested step and for each prognostic field, the relative L2 and max-norm
error of the mixed form against the FP64 form, the error relative to the
field's variability (its standard deviation; v starts at zero, so its
plain relative error divides by a small norm), and the relative change of
the total mass of each form since step 0.  Norms are taken on the device in
FP64.
"""
from __future__ import annotations

import argparse
import json
import time

import torch

from . import ic
from .dycore import Dycore

NAMES = ('dp', 'pt', 'ud', 'vd')


def fields(dyn, shape):
    """Interior of the four fields as FP64 tensors (the library runs on its
    own stream: synchronise on both sides of the copies)."""
    out = {}
    torch.cuda.synchronize()
    for n in NAMES:
        t = torch.empty(shape, dtype=torch.float64, device='cuda')
        torch.cuda.synchronize()
        dyn.download_device(n, t)
        out[n] = t
    dyn.sync()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('--n', type=int, default=2048)
    ap.add_argument('--nlay', type=int, default=64)
    ap.add_argument('--steps', default='50,100,200')
    ap.add_argument('--seed', type=int, default=1)
    ap.add_argument('--dt', type=float, default=30.0)
    ap.add_argument('--remap-every', type=int, default=8)
    args = ap.parse_args(argv)
    marks = sorted(int(s) for s in args.steps.split(','))
    torch.cuda.set_device(0)
    st = ic.jet_case(args.n, args.n, args.nlay, 25e3, 25e3, seed=args.seed)
    ref = Dycore(st, 'fp64')
    mix = Dycore(st, 'mixed')
    shape = (st.nlay, st.ny, st.nx)
    m0 = {'fp64': ref.mass(), 'mixed': mix.mass()}
    report = {'workload': 'jet %dx%dx%d (seed %d), dt %g s, remap every %d' % (
        args.n, args.n, args.nlay, args.seed, args.dt, args.remap_every), 'steps': {}}
    t0 = time.time()
    step = 0
    for mark in marks:
        while step < mark:
            step += 1
            r = step % args.remap_every == 0
            ok_r = ref.step(args.dt, remap=r, check_stable=False)
            ok_m = mix.step(args.dt, remap=r, check_stable=False)
        a, b = fields(ref, shape), fields(mix, shape)
        entry = {'stable_fp64': ref.check_stability(), 'stable_mixed': mix.check_stability()}
        for n in NAMES:
            d = b[n] - a[n]
            entry[n] = {
                'rel_l2': (d.norm() / a[n].norm()).item(),
                'rel_max': (d.abs().max() / a[n].abs().max()).item(),
                'rel_l2_to_std': (d.norm() / ((a[n] - a[n].mean()).norm())).item(),
            }
        entry['mass_rel_change'] = {'fp64': ref.mass() / m0['fp64'] - 1.0, 'mixed': mix.mass() / m0['mixed'] - 1.0}
        report['steps'][str(mark)] = entry
        del a, b
    report['wall_s'] = time.time() - t0
    print(json.dumps(report))
    return report


if __name__ == '__main__':
    main()
