"""Small GPU cases of the project's kernels, sized for an ncu capture: a few GB
on the device at most (inputs larger than the 126 MB L2, so DRAM counters
mean something) and a handful of launches, so that a capture of one launch
ends by itself in a minute or two.  Run the same command without ncu first.

    python -m openifs_b200.profile_cases cloudsc --blocks 518 [--precision 0]
        one batched CLOUDSC call over 518 NPROMA blocks of 128 (66,304
        columns: one wave of 148 CTAs x 448 columns), seed 2
    python -m openifs_b200.profile_cases satadj --blocks 256 --repeat 3
        CLOUD_SATADJ over 256 blocks of 128, seed 2, called 3 times
    python -m openifs_b200.profile_cases conv5 --columns 8192 --repeat 2
        the surrogate's 5-tap level convolution (width 128, SiLU and
        residual epilogue) on 8,192 columns x 144 rows, called twice
    python -m openifs_b200.profile_cases surrogate --blocks 256 --repeat 2
        the guarded surrogate (committed width-128 weights: input
        preparation, network, guard, FP64 fallback of the flagged columns)
        over 256 NPROMA blocks of 128 (32,768 columns), seed 2, run twice

Each prints "ok" and exits 0 when the case ran.
"""
import argparse

KLEV = 137
PTSPHY = 3600.0
SEED = 2


def run_cloudsc(blocks, precision, nproma=128):
    import torch
    from . import cloudsc, inputs
    p = cloudsc.default_params()
    cloudsc.setup(p)
    arrs = inputs.generate(blocks, nproma, p, seed=SEED)
    d = {k: torch.from_numpy(v).cuda() for k, v in arrs.items()}
    cloudsc.cloudsc_batched(p, d, nproma, KLEV, blocks, nproma * blocks, PTSPHY, precision=precision)
    torch.cuda.synchronize()


def run_satadj(blocks, repeat, nproma=128):
    import torch
    from . import cloudsc, inputs
    p = cloudsc.default_params(PTSPHY, inputs.ncldtop_l137())
    host = inputs.generate_satadj(blocks, nproma, p, seed=SEED)
    d = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    cloudsc.setup(p)
    for _ in range(repeat):
        cloudsc.satadj_batched(p, d, nproma, KLEV, blocks, nproma * blocks, PTSPHY)
    torch.cuda.synchronize()


def run_conv5(columns, repeat, width=128, lp=144):
    import torch
    from . import tcgemm
    rows = columns * lp
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.randn(rows, width, device="cuda", generator=g).bfloat16()
    w5 = (torch.randn(5, width, width, device="cuda", generator=g) * 0.02).bfloat16()
    out = torch.empty(rows, width, device="cuda", dtype=torch.bfloat16)
    b = torch.zeros(width, device="cuda")
    tcgemm.set_impl(0)
    for _ in range(repeat):
        tcgemm.conv_gemm(a, w5, tcgemm.EPI_SILU, width, 5, lp, KLEV, b, out, None, a)
    torch.cuda.synchronize()


def run_surrogate(blocks, repeat, nproma=128):
    import torch
    from . import cloudsc, inputs, surrogate as S
    p = cloudsc.default_params()
    cloudsc.setup(p)
    host = inputs.generate(blocks, nproma, p, seed=SEED)
    d = {k: torch.from_numpy(v).cuda() for k, v in host.items()}
    net = S.Net.load(S.WEIGHTS)
    run = S.Runner(net, p, nproma, blocks, capacity=nproma * blocks // 16)
    b = run.prepare(d)
    for _ in range(repeat):
        run.run(b)
    torch.cuda.synchronize()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["cloudsc", "satadj", "conv5", "surrogate"])
    ap.add_argument("--blocks", type=int, default=None)
    ap.add_argument("--columns", type=int, default=8192)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=None)
    a = ap.parse_args(argv)
    if a.case == "cloudsc":
        run_cloudsc(a.blocks or 518, a.precision)
    elif a.case == "satadj":
        run_satadj(a.blocks or 256, a.repeat or 3)
    elif a.case == "surrogate":
        run_surrogate(a.blocks or 256, a.repeat or 2)
    else:
        run_conv5(a.columns, a.repeat or 2)
    print("ok")


if __name__ == "__main__":
    main()
