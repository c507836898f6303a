"""The ``tccg`` command for B200: ``python -m tccg_b200 file.tccg [flags]``.

Flags follow TCCG's argparse surface (tccg.py:1253-1284). Kept with their
meaning: ``--floatType s|d``, ``--maxImplementations N`` (-1 = no bound),
``--maxImplementationsTTGT``, ``--ignoreDatabase``, ``--generateOnly`` (emit
without tuning), ``--gettOnly`` / ``--noGETT`` / ``--noTTGT`` / ``--noLoG``,
``--testing`` (check the tuned kernel; TCCG compares against its loop nest,
tccg.py:1010-1050 -- here against the library's FP64 path with TCCG's
``equal()`` tolerance, sign-aware), ``--maxWorkspace`` (GB), ``--verbose``,
``--keep`` (keep nothing else to clean: accepted). Accepted and ignored
because they configure TCCG's CPU build: ``--numThreads``, ``--affinity``,
``--compiler``, ``--noBatchedGEMM``, ``--timePacking``, ``--useDynamicMemory``,
``--fastMeasurements``, ``--noGEMM``; ``--arch`` must be ``sm_100a`` (or
``cuda``), ``--useTCL`` is rejected. New: ``--precision
fp32|fp64|bf16|bf16x3`` and ``--outdir``.
"""
from __future__ import annotations

import argparse
import sys

from .spec import TccgSyntaxError, TccgUnsupported, parse_file


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="tccg",
                                description="Generate B200 (sm_100a) code for a tensor contraction.")
    p.add_argument("filename")
    for flag in ("--verbose", "--testing", "--keep", "--noBatchedGEMM", "--generateOnly",
                 "--gettOnly", "--noGETT", "--noLoG", "--noGEMM", "--noTTGT", "--useTCL",
                 "--useDynamicMemory", "--timePacking", "--ignoreDatabase", "--fastMeasurements"):
        p.add_argument(flag, action="store_true")
    p.add_argument("--numThreads", type=int)
    p.add_argument("--maxImplementations", type=int, default=16)
    p.add_argument("--maxImplementationsTTGT", type=int, default=1)
    p.add_argument("--maxImplementationsLoG", type=int, default=1)
    p.add_argument("--maxWorkspace", type=float)
    p.add_argument("--arch", default="sm_100a")
    p.add_argument("--compiler")
    p.add_argument("--floatType", default="s")
    p.add_argument("--affinity")
    p.add_argument("--precision", choices=["fp32", "fp64", "bf16", "bf16x3"])
    p.add_argument("--outdir", default="tccg_implementations")
    return p


def settings_banner(args, con) -> str:
    lines = ["-----------------SETTINGS-----------------",
             "Version".ljust(20) + "tccg_b200 0.1",
             "inputfile".ljust(20) + args.filename,
             "maxImplementations".ljust(20) + str(args.maxImplementations),
             "architecture".ljust(20) + "sm_100a (B200)",
             "floatType".ljust(20) + {"s": "float", "d": "double"}[args.floatType],
             "precision".ljust(20) + str(args.precision),
             "------------------------------------------"]
    return "\n".join(lines)


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    if args.floatType not in ("s", "d"):
        print("ERROR: floatType %s is not supported yet." % args.floatType, file=sys.stderr)
        return 2
    if args.useTCL:
        print("ERROR: --useTCL: TCL is not part of this build.", file=sys.stderr)
        return 2
    if args.arch not in ("sm_100a", "cuda", "b200"):
        print("ERROR: --arch: only sm_100a (B200) is generated.", file=sys.stderr)
        return 2
    args.precision = args.precision or {"s": "fp32", "d": "fp64"}[args.floatType]
    if (args.floatType == "d") != (args.precision == "fp64"):
        print("ERROR: --floatType=%s does not go with --precision=%s" % (args.floatType, args.precision),
              file=sys.stderr)
        return 2
    try:
        con = parse_file(args.filename)
        con.validate()
    except (TccgSyntaxError, TccgUnsupported) as e:
        print("ERROR: %s" % e, file=sys.stderr)
        return 1
    print(settings_banner(args, con))
    print(str(con))
    print("m: %d\nn: %d\nk: %d" % (con.sizeM, con.sizeN, con.sizeK))

    from .plan import Tuning
    methods = []
    if not args.noGETT:
        methods.append("gett")
    if not (args.noTTGT or args.gettOnly):
        methods.append("ttgt")
    if not methods:
        print("ERROR: every method is disabled", file=sys.stderr)
        return 2
    if args.generateOnly or args.maxImplementations == 0:
        tuning = Tuning(method=methods[0])
    else:
        from .autotune import autotune
        tuning = autotune(con, args.precision, args.maxImplementations,
                          ignore_cache=args.ignoreDatabase, methods=tuple(methods),
                          verbose=args.verbose, max_workspace_gb=args.maxWorkspace)
    print("Best candidate: %s" % tuning.key())

    if args.testing:
        ok = _testing(con, args.precision, tuning)
        if not ok:
            print("ERROR: version '%s' failed" % tuning.key())
            return 1

    from .emit import emit
    paths = emit(con, args.precision, tuning, args.floatType, args.outdir)
    print("The generated code is available at: %s" % paths["cu"])
    return 0


def _testing(con, precision, tuning) -> bool:
    """TCCG's --testing: the tuned kernel against a reference on TCCG's
    deterministic inputs (tccg.py:957-971), with equal()'s tolerance (1e-4
    float, 1e-9 double; tccg.py:869-873), differences taken with their sign."""
    import torch
    from .plan import Plan
    dev = torch.device("cuda", torch.cuda.current_device())

    def init(n, o, m, dt):
        i = torch.arange(n, dtype=torch.int64, device=dev)
        return (((10 + ((i + o) * m) % 100).float()) / 110.0).to(dt)

    dt = torch.float64 if precision == "fp64" else torch.float32
    A = init(con.A0.num_elements(), 1, 17, dt)
    B = init(con.B0.num_elements(), 2, 3, dt)
    C0 = init(con.C0.num_elements(), 3, 13, dt)
    C = C0.clone()
    Plan(con, precision=precision, tuning=tuning).run(A, B, C)
    R = C0.double().clone()
    Plan(con, precision="fp64").run(A.double(), B.double(), R)
    torch.cuda.synchronize()
    d = (C.double() - R).abs()
    mx = torch.maximum(C.double().abs(), R.abs()).clamp_min(1e-300)
    crit = torch.minimum(d, d / mx)
    tol = 1e-9 if precision == "fp64" else 1e-4
    worst = crit.max().item()
    print("testing: worst min(abs, rel) error %.3e (tolerance %.0e)" % (worst, tol))
    return worst <= tol


if __name__ == "__main__":
    sys.exit(main())
