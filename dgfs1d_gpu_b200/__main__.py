"""Command line of the drivers, as the reference's console scripts take it.

    python -m dgfs1d_gpu_b200 dgfsStd1D run cfg.ini [-v mesh::Ne 8 ...]
    python -m dgfs1d_gpu_b200 dgfsStd1D restart cfg.ini dist.npz_rank=0 [-v ...]

Drivers: dgfsStd1D, dgfsBi1D, dgfsAstd1D, dgfsABstd1D, dgfsABUstd1D, dgfsABE2std1D
(setup.py:91-107 of the reference; each there is ``<driver> run|restart``,
dgfs1D/initialize.py:7-50).  ``-v section::key value`` overrides an INI
value.  One rank: ``restart`` takes one distribution file.  The run marches
to ``[time-integrator] tend`` with the writers the INI enables and prints the
step count and the elapsed time as the reference does.
"""
import argparse
import sys
import time

from .config import Config

DRIVERS = {
    'dgfsStd1D': ('std.solver', 'DGFSStd1D'),
    'dgfsBi1D': ('bi.solver', 'DGFSBi1D'),
    'dgfsAstd1D': ('astd.solver', 'DGFSAstd1D'),
    'dgfsABstd1D': ('astd.solver', 'DGFSABstd1D'),
    'dgfsABUstd1D': ('astd.solver', 'DGFSABUstd1D'),
    'dgfsABE2std1D': ('astd.solver', 'DGFSABE2std1D'),
}


def parse(argv):
    ap = argparse.ArgumentParser(prog='python -m dgfs1d_gpu_b200')
    ap.add_argument('driver', choices=sorted(DRIVERS))
    sp = ap.add_subparsers(dest='cmd', required=True)
    for name in ('run', 'restart'):
        p = sp.add_parser(name)
        p.add_argument('inp', help='input file')
        if name == 'restart':
            p.add_argument('dist', nargs='+', help='distribution file (one per rank)')
        p.add_argument('-v', nargs=2, action='append', default=[],
                       metavar=('SECTION::KEY', 'VALUE'),
                       help='substitute a value, e.g. -v mesh::Ne 4')
    return ap.parse_args(argv)


def make_solver(args):
    import importlib
    mod, cls = DRIVERS[args.driver]
    solver_cls = getattr(importlib.import_module('.' + mod, __package__), cls)
    cfg = Config.load(args.inp, defaults=Config.overrides(args.v))
    if args.cmd == 'restart':
        if len(args.dist) != 1:
            raise SystemExit('No. of distributions != nranks (one rank)')
        return solver_cls(cfg, restart=args.dist[0])
    return solver_cls(cfg)


def main(argv=None):
    args = parse(sys.argv[1:] if argv is None else argv)
    s = make_solver(args)
    t0 = time.perf_counter()
    s.run()
    import torch
    torch.cuda.synchronize()
    print('Nsteps', s.nsteps, ', elapsed time', time.perf_counter() - t0, 's')
    return s


if __name__ == '__main__':
    main()
