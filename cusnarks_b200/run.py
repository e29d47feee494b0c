"""Run one synthetic workload of the prover path and print its device times.

    python -m cusnarks_b200.run msm   --log-n 20 [--g2] [--fixed] [--window C] [--reps K]
    python -m cusnarks_b200.run prove --log-m 20 [--no-fixed] [--batch B] [--reps K]
    python -m cusnarks_b200.run ntt   --log-n 20 [--hstep reference|coset] [--reps K]

Inputs are seeded: MSM scalars uniform in Fr, bases k_i * G (k_i seeded, built on the GPU);
prove runs the synthetic R1CS family of the benchmark (3 nonzeros per A/B row) with a key
from seeded toxic waste.  One untimed call warms up, then K calls run inside a CUDA
profiler range (cudaProfilerStart/Stop), so a profiler started with its capture off (ncu
--profile-from-start off) sees exactly those K calls.  One JSON line per call: device ms
(CUDA events on the launching stream) and, for an MSM, the bucket-accumulation ms.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _msm(args, ctx):
    import torch
    from .synth import random_field, g1_generator, g2_generator
    n = 1 << args.log_n
    pw = 32 if args.g2 else 16
    rng = np.random.Generator(np.random.PCG64(args.seed))
    dev = torch.device("cuda", ctx.device)
    d_k = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    d_s = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    g = torch.from_numpy((g2_generator() if args.g2 else g1_generator()).view(np.int32)).to(dev)
    d_p = torch.empty((n, pw), dtype=torch.int32, device=dev)
    d_out = torch.zeros(pw, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    ctx.scmul_device(d_k.data_ptr(), g.data_ptr(), n, d_p.data_ptr(), ec2=args.g2, point_stride_words=0)
    ctx.sync()
    if args.fixed:
        c = args.window or ctx.msm_fixed_window(n, args.g2)
        table = torch.empty(ctx.msm_fixed_table_points(n, c) * pw, dtype=torch.int32, device=dev)
        ctx.msm_fixed_table_device(d_p.data_ptr(), n, c, table.data_ptr(), ec2=args.g2)
        ctx.sync()

        def call():
            ctx.msm_fixed_device(d_s.data_ptr(), table.data_ptr(), n, c, d_out.data_ptr(), ec2=args.g2)
    else:
        from ._lib import lib
        c = args.window or int(lib().cs_msm_default_window(n, int(args.g2)))

        def call():
            ctx.msm_device(d_s.data_ptr(), d_p.data_ptr(), n, d_out.data_ptr(), ec2=args.g2, window=c)

    info = {"workload": "msm", "group": "G2" if args.g2 else "G1", "log_n": args.log_n,
            "variant": "fixed-base" if args.fixed else "generic", "window": c}
    return call, info


def _prove(args, ctx):
    import torch
    from .groth import SyntheticCircuit, setup_pk, Prover
    from .synth import to_limbs
    circ = SyntheticCircuit(ctx, args.log_m, seed=args.seed)
    pk = setup_pk(ctx, circ, seed=args.seed + 1)
    prover = Prover(ctx, pk, fixed_base=-1 if args.no_fixed else 0)
    if not args.graphs:  # stage times need the launches themselves (graph replays carry none)
        ctx.set_prove_graphs(False)
    r, s = to_limbs(0x1234567890abcdef), to_limbs(0xfedcba0987654321)
    dev = torch.device("cuda", ctx.device)
    info = {"workload": "prove", "log_m": args.log_m, "fixed_windows": prover.fixed_windows()}
    if args.batch > 1:  # B proofs of the same witness buffer with distinct r, s in one pass
        d_proofs = torch.zeros((args.batch, 64), dtype=torch.int32, device=dev)
        rs = [to_limbs(0x1234567890abcdef + i) for i in range(args.batch)]
        ss = [to_limbs(0xfedcba0987654321 + i) for i in range(args.batch)]
        torch.cuda.synchronize()

        def call():
            prover.prove_batch_device([circ.d_w.data_ptr()] * args.batch, rs, ss,
                                      [d_proofs[i].data_ptr() for i in range(args.batch)])

        info["batch"] = args.batch
        call.keep = (circ, pk, prover, d_proofs)
        return call, info
    d_proof = torch.zeros(64, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def call():
        prover.prove_device(circ.d_w.data_ptr(), r, s, d_proof.data_ptr())

    call.keep = (circ, pk, prover, d_proof)
    return call, info


def _ntt(args, ctx):
    import torch
    from .synth import random_field
    n = 1 << args.log_n
    rng = np.random.Generator(np.random.PCG64(args.seed))
    dev = torch.device("cuda", ctx.device)
    a = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    b = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    c = torch.from_numpy(random_field(rng, n).view(np.int32)).to(dev)
    out = torch.empty(2 * n * 8, dtype=torch.int32, device=dev)  # 2m coefficients (reference variant)
    torch.cuda.synchronize()
    if args.hstep:
        variant = 0 if args.hstep == "reference" else 1

        def call():
            ctx.hstep_device(variant, a.data_ptr(), b.data_ptr(), c.data_ptr(), args.log_n, out.data_ptr())
        info = {"workload": "hstep", "variant": args.hstep, "log_m": args.log_n}
    else:
        def call():
            ctx.ntt_device(a.data_ptr(), out.data_ptr(), args.log_n, 1)
        info = {"workload": "ntt", "direction": "forward", "log_n": args.log_n}
    call.keep = (a, b, c, out)
    return call, info


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m cusnarks_b200.run")
    sub = ap.add_subparsers(dest="what", required=True)
    m = sub.add_parser("msm")
    m.add_argument("--log-n", type=int, default=20)
    m.add_argument("--g2", action="store_true")
    m.add_argument("--fixed", action="store_true", help="fixed-base tables (built before timing)")
    m.add_argument("--window", type=int, default=0)
    p = sub.add_parser("prove")
    p.add_argument("--log-m", type=int, default=20)
    p.add_argument("--no-fixed", action="store_true", help="generic MSMs instead of fixed-base tables")
    p.add_argument("--graphs", action="store_true", help="replay the proof as a CUDA graph (no stage times)")
    p.add_argument("--batch", type=int, default=1,
                   help="B proofs with the key in one pass (cs_prove_batch_device, a CUDA graph); ms per pass")
    t = sub.add_parser("ntt")
    t.add_argument("--log-n", type=int, default=20)
    t.add_argument("--hstep", choices=["reference", "coset"], default=None)
    for q in (m, p, t):
        q.add_argument("--reps", type=int, default=3)
        q.add_argument("--seed", type=int, default=100)
        q.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    import torch
    from .context import Context
    torch.cuda.set_device(args.device)
    ctx = Context(args.device)
    call, info = {"msm": _msm, "prove": _prove, "ntt": _ntt}[args.what](args, ctx)
    call()
    ctx.sync()
    torch.cuda.profiler.start()
    for i in range(args.reps):
        call()
        ctx.sync()
        rec = dict(info, rep=i, ms=round(ctx.last_ms, 4))
        if args.what == "msm":
            rec["accumulate_ms"] = round(ctx.last_phase_ms, 4)
        if args.what == "prove" and not args.graphs and args.batch <= 1:
            rec["stages_ms"] = call.keep[2].stages()
        print(json.dumps(rec), flush=True)
    torch.cuda.profiler.stop()


if __name__ == "__main__":
    main()
