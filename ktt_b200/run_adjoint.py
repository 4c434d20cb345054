"""Time the charge-fitting step: forward map, adjoint gradient, and one autograd training step.

    python -m ktt_b200.run_adjoint [--repeat 5] [--n 128] [--atoms 8192]

8,192 atoms uniform in a 64 A cube, 128^3 grid at 0.5 A; the loss 0.5 sum w (V - V*)^2 with the
1.5 A exclusion weights.  Prints one JSON line: device time and pair rate of the forward map in
FP32 and FP64-merge forms and of the adjoint kernel (including its chunk reduction), and the wall
time of one loss.backward() + Adam step through the autograd function.
"""
from __future__ import annotations

import argparse
import json
import time


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=5)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--atoms", type=int, default=8192)
    args = ap.parse_args()

    import torch

    import ktt_b200
    from ktt_b200 import workloads

    box = args.n * 0.5
    atoms_np, q_target, dims, h, excl = workloads.adjoint_problem(n_atoms=args.atoms, n=args.n, box=box)
    weight = torch.from_numpy(workloads.exclusion_weights(atoms_np, dims, h, excl)).cuda()
    ctx = ktt_b200.CoulombContext(0)
    atoms = torch.from_numpy(atoms_np).cuda()
    pairs = float(dims[0] * dims[1] * dims[2] * args.atoms)
    out = {"dims": list(dims), "atoms": args.atoms, "pairs": pairs}

    def timed(fn):
        fn()
        ctx.synchronize()
        ms = []
        for _ in range(args.repeat):
            fn()
            ms.append(ctx.elapsed_ms())
        ctx.synchronize()
        return min(ms)

    fwd_fp32 = ktt_b200.Tune(z_iterations=8, x_points=2, unroll=2, rsqrt_soft=2)
    fwd_fp64 = ktt_b200.Tune(z_iterations=8, x_points=2, precision=ktt_b200.PREC_FP64_MERGE, rsqrt_soft=2)
    for name, tune in (("forward_fp32", fwd_fp32), ("forward_fp64_merge", fwd_fp64)):
        ms = timed(lambda: ctx.forward_3d(atoms, dims, h, tune=tune))
        out[name] = {"ms": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9}
    target_atoms = atoms_np.copy()
    target_atoms[:, 3] = q_target
    target = ctx.forward_3d(torch.from_numpy(target_atoms).cuda(), dims, h, tune=fwd_fp64)
    v = ctx.forward_3d(atoms, dims, h, tune=fwd_fp64)
    grad_map = (weight * (v - target)).contiguous()
    ms = timed(lambda: ktt_b200.adjoint_3d(ctx, atoms, dims, h, grad_map))
    out["adjoint"] = {"ms": ms, "gpairs_per_s": pairs / (ms * 1e-3) / 1e9}

    q = atoms[:, 3].clone().requires_grad_(True)
    xyz = atoms[:, :3].clone()
    opt = torch.optim.Adam([q], lr=0.005)

    def step():
        opt.zero_grad()
        vv = ktt_b200.coulomb_map(torch.cat([xyz, q[:, None]], dim=1), ctx, dims, h, None, fwd_fp64)
        loss = 0.5 * (weight * (vv - target) ** 2).sum()
        loss.backward()
        opt.step()
        return loss

    step()
    torch.cuda.synchronize()
    wall = []
    for _ in range(args.repeat):
        t0 = time.perf_counter()
        step()
        torch.cuda.synchronize()
        wall.append((time.perf_counter() - t0) * 1e3)
    out["train_step_ms"] = min(wall)
    print(json.dumps(out))
    ctx.close()


if __name__ == "__main__":
    main()
