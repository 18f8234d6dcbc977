"""Train the learned stage on residual / error pairs that the GMG solver
itself generates, with this package's own convolution kernels, then evaluate
it as a flexible-CG stage against the solver without it.

Data.  Seeded two-material noise parts (``generators.two_material_part``:
blurred-noise geometry, z=0 face clamped, a second noise field splitting
steel / ABS) of 64..128 voxels per axis, each with one random load case
(``generators.load_cases``: direction uniform on the sphere, 1-10 kN on a
random 8x8 top patch).  Per part the mixed-precision solver solves for the
displacement u, and the error of the V-cycle iteration started from zero,
e_j = (I - M A)^j u (M = one FP32 V-cycle), gives the pairs
(r_j = A e_j, e_j), j in SNAPSHOTS: the residual the stage sees after the
V-cycle inside the flexible CG, and the error it should remove.  Late
snapshots are dominated by the slow modes of the V-cycle -- the ones the
Krylov iteration spends its iterations on.

Loss.  The solver scales the stage's correction c = P^L (mask_L * y) (P =
trilinear node interpolation, the V-cycle's prolongation) by the A-norm-
optimal step, so only its direction matters: the loss is 1 - cos^2(c, e_j)
over the free fine DOFs.

Usage (one GPU):
    python -m voxelsim_fea_b200.learned.train --parts 2000 --out unet_weights.npz
"""

import argparse
import json
import math
import multiprocessing as mp
import os
import time

import numpy as np

SIZES = (64, 80, 96, 112, 128)
SNAPSHOTS = (2, 8, 24)


def part_spec(seed, sizes=SIZES):
    rng = np.random.default_rng(seed)
    shape = tuple(int(rng.choice(sizes)) for _ in range(3))
    return shape, float(rng.uniform(3.0, 5.0))


def make_part(seed, sizes=SIZES, shape=None, drop_islands=False):
    """CPU-only geometry / load generation (runs in worker processes).
    ``drop_islands``: pass the part through the reference's island step
    (``generators.drop_unsupported``) before placing its load, as every job
    of the reference is before its solve."""
    from .. import generators
    spec_shape, sigma = part_spec(seed, sizes)
    shape = shape or spec_shape
    prob = generators.two_material_part(shape, seed=seed, sigma=sigma)
    if drop_islands:
        prob = generators.drop_unsupported(prob)
    f = generators.load_cases(prob, 1, seed + 1)[0]
    E = np.where(prob["active"], prob["E_stiff"], prob["E_stiff"] * 1e-9)
    return {"seed": seed, "dims": shape, "E": E, "nu": np.asarray(prob["nu"], dtype=float),
            "fixed": prob["fixed_dofs"], "f": f}


def _make_part_star(a):
    return make_part(*a)


class Pair:
    __slots__ = ("inp", "scale", "eref", "e", "mask0", "maskL", "dimsL", "dims0")


def _bits(mask_u8, shape):
    import torch
    m = torch.as_tensor(mask_u8.astype(np.int64), device="cuda")
    bits = torch.stack([(m >> c) & 1 for c in range(3)], dim=-1).to(torch.float32)
    return bits.view(*shape, 3)


def solver_for(part, **opt):
    from ..multigrid import MGSolver, SolverOptions
    nx, ny, nz = part["dims"]
    return MGSolver(nx, ny, nz, part["fixed"], nu=0.3, options=SolverOptions.fast(**opt))


def propagate(m, e, n):
    """(I - M A)^n e on the device (vf_mg_propagate)."""
    from .. import _lib
    out = np.empty(m.ndof)
    ee = _lib.f64(e)
    _lib.check(_lib.load().vf_mg_propagate(m._handle(), _lib.ptr(ee), int(n), _lib.ptr(out)), m._h, "propagate")
    return out


def make_pairs(part, level=1, snapshots=SNAPSHOTS):
    """Residual / error pairs of one part (see the module docstring)."""
    import torch
    from . import stage
    m = solver_for(part)
    try:
        # any displacement-like field seeds the error sequence: a loose solve
        u = m.solve(part["E"], part["f"], tol=1e-3, max_cg=300, nu_elem=part["nu"])
        stage.configure(m, None, level, False)
        nx, ny, nz = part["dims"]
        lx, ly, lz = m.levels[level]["dims"]
        mask0 = _bits(m.levels[0]["free"].reshape(-1, 3).astype(np.uint8) @ np.array([1, 2, 4], dtype=np.uint8),
                      (nz + 1, ny + 1, nx + 1))
        maskL = _bits(stage.level_mask(m, level), (lz + 1, ly + 1, lx + 1))
        out = []
        e = u
        done = 0
        for j in snapshots:
            e = propagate(m, e, j - done)
            done = j
            r = m._apply(0, e)
            rL = r
            for li in range(level):
                rL = m._restrict(li, rL)
            p = Pair()
            p.inp, p.scale, p.eref = stage.make_input(m, rL)
            p.e = torch.as_tensor(e.reshape(nz + 1, ny + 1, nx + 1, 3), dtype=torch.float32, device="cuda")
            p.mask0, p.maskL = mask0, maskL
            p.dimsL = (lz + 1, ly + 1, lx + 1)
            p.dims0 = (nz + 1, ny + 1, nx + 1)
            out.append(p)
        return out
    finally:
        m.close()


def predict_fine(net, p):
    """The stage's fine-grid correction for pair p (training form)."""
    import torch.nn.functional as F
    y = net(p.inp)
    zl, yl, xl = p.dimsL
    yL = y[:zl, :yl, :xl, :3] * (p.scale / p.eref) * p.maskL
    ef = F.interpolate(yL.permute(3, 0, 1, 2).unsqueeze(0), size=p.dims0, mode="trilinear", align_corners=True)
    return ef.squeeze(0).permute(1, 2, 3, 0) * p.mask0


def pair_loss(net, p):
    """1 - cos^2 between the stage's correction and the error (scale-free)."""
    c = predict_fine(net, p)
    e = p.e / p.e.norm().clamp_min(1e-300)
    ce = (c * e).sum()
    return 1.0 - ce * ce / (c * c).sum().clamp_min(1e-30)


def train(parts=2000, level=1, snapshots=SNAPSHOTS, steps_per_part=3, buffer_cap=256, lr=1e-3, seed=0, workers=16,
          log_every=50, sizes=SIZES, verbose=True):
    import torch
    from .unet import UNet
    ctx = mp.get_context("spawn")
    seeds = [1_000_000 + seed * 100_003 + 17 * i for i in range(parts)]
    rng = np.random.default_rng(seed)
    total_steps = parts * steps_per_part
    hist = []
    t0 = time.time()
    with ctx.Pool(workers) as pool:
        torch.manual_seed(seed)
        net = UNet(seed).cuda()
        opt = torch.optim.Adam(net.parameters(), lr=lr)
        sched = torch.optim.lr_scheduler.LambdaLR(
            opt, lambda s: 0.02 + 0.98 * 0.5 * (1 + math.cos(math.pi * min(s, total_steps) / total_steps)))
        buf = []
        run = []
        for i, part in enumerate(pool.imap(_make_part_star, [(s, sizes) for s in seeds], chunksize=2)):
            buf.extend(make_pairs(part, level, snapshots))
            if len(buf) > buffer_cap:
                del buf[:len(buf) - buffer_cap]
            for _ in range(steps_per_part):
                p = buf[int(rng.integers(len(buf)))]
                loss = pair_loss(net, p)
                opt.zero_grad(set_to_none=True)
                loss.backward()
                opt.step()
                sched.step()
                run.append(float(loss.detach()))
            if (i + 1) % log_every == 0 or i + 1 == parts:
                m = float(np.mean(run[-log_every * steps_per_part:]))
                hist.append((i + 1, m))
                if verbose:
                    print(f"[train] parts {i + 1}/{parts}  loss {m:.4f}  {time.time() - t0:.0f}s", flush=True)
    return net, hist, time.time() - t0


def eval_configs():
    """(name, SolverOptions, learned stage on) of the evaluation."""
    from ..multigrid import SolverOptions
    return (("plain_fp64", SolverOptions.robust(), False),
            ("learned_fp64", SolverOptions.robust(), True),
            ("mixed", SolverOptions.fast(), False),
            ("mixed_reliable", SolverOptions.fast(mixed_mode="reliable"), False),
            ("mixed_restart", SolverOptions.fast(mixed_mode="restart", inner_tol=1e-4), False),
            ("learned_mixed_restart", SolverOptions.fast(mixed_mode="restart", inner_tol=1e-4), True),
            ("learned_mixed", SolverOptions.fast(), True))


def headline_configs():
    """The headline comparison: plain FP64 GMG-PCG, mixed, learned + mixed."""
    from ..multigrid import SolverOptions
    return (("plain_fp64", SolverOptions.robust(), False),
            ("mixed", SolverOptions.fast(), False),
            ("learned_mixed", SolverOptions.fast(), True))


def modes_configs():
    """Plain FP64 against the mixed-precision forms: FP32 CG with residual
    replacement, FP64 PCG around the FP32 V-cycle, and the latter with the
    learned stage."""
    from ..multigrid import SolverOptions
    return (("plain_fp64", SolverOptions.robust(), False),
            ("mixed_reliable", SolverOptions.fast(mixed_mode="reliable"), False),
            ("outer64", SolverOptions.fast(mixed_mode="outer64"), False),
            ("learned_outer64", SolverOptions.fast(mixed_mode="outer64"), True))


def evaluate(params, level, seeds, shape, tol=1e-8, verbose=True, configs=None, max_cg=None,
             drop_islands=True):
    """Solve held-out parts without and with the learned stage (FP64 and
    mixed precision); per-part iterations and device times.  ``max_cg``
    None is the reference's cap of 1000 iterations; ``drop_islands`` runs
    each part through the reference's island step first."""
    from ..multigrid import MGSolver
    from . import stage
    rows = []
    configs = configs or eval_configs()
    for s in seeds:
        part = make_part(s, shape=shape, drop_islands=drop_islands)
        nx, ny, nz = part["dims"]
        row = {"seed": s, "active_voxels": int(np.count_nonzero(part["E"] > part["E"].max() * 1e-6))}
        for name, opts, use in configs:
            m = MGSolver(nx, ny, nz, part["fixed"], nu=0.3, options=opts)
            m.set_density(part["E"], nu_elem=part["nu"])
            if use:
                stage.configure(m, params, level, True)
            m.solve(part["E"], part["f"], tol=tol, nu_elem=part["nu"], max_cg=max_cg)   # warm (graph capture)
            m.solve(part["E"], part["f"], tol=tol, nu_elem=part["nu"], max_cg=max_cg)
            inf = m.last_info
            row[name] = {"iters": int(inf.iters), "solve_ms": float(inf.device_ms),
                         "true_resid": float(inf.true_resid), "converged": bool(inf.converged)}
            if use:   # iteration at which the stage was switched off for stagnating (0: stayed on)
                row[name]["stage_off_at"] = int(inf.outer_iters)
            m.close()
        rows.append(row)
        if verbose:
            print(f"[eval] seed {s}: " + "  ".join(f"{k} {row[k]['iters']} it {row[k]['solve_ms']:.0f} ms"
                                                  for k, _, _ in configs), flush=True)
    return rows


def summarize(rows, configs):
    """Per configuration: parts converged, mean / median iterations and
    device solve time, and the summed solve time."""
    out = {}
    for k, _, _ in configs:
        it = [r[k]["iters"] for r in rows]
        ms = [r[k]["solve_ms"] for r in rows]
        out[k] = {"converged": int(sum(r[k]["converged"] for r in rows)), "parts": len(rows),
                  "iters_mean": float(np.mean(it)), "iters_median": float(np.median(it)),
                  "solve_ms_mean": float(np.mean(ms)), "solve_ms_median": float(np.median(ms)),
                  "solve_ms_total": float(np.sum(ms))}
        offs = [r[k]["stage_off_at"] for r in rows if "stage_off_at" in r[k]]
        if offs:
            out[k]["stage_switched_off"] = int(sum(1 for v in offs if v > 0))
    return out


def _report(rows, configs, args):
    summary = summarize(rows, configs)
    print(json.dumps(summary), flush=True)
    if args.eval_json:
        with open(args.eval_json, "w") as fh:
            json.dump({"protocol": {"size": args.eval_size, "parts": args.eval, "tol": 1e-8,
                                    "max_cg": args.max_cg or 1000,
                                    "islands": "kept (26-connected)" if args.raw_parts else
                                    "dropped by the reference's island step"},
                       "rows": rows, "summary": summary}, fh, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--parts", type=int, default=2000)
    ap.add_argument("--level", type=int, default=1)
    ap.add_argument("--snapshots", type=str, default=",".join(map(str, SNAPSHOTS)))
    ap.add_argument("--steps-per-part", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--sizes", type=str, default=",".join(map(str, SIZES)))
    ap.add_argument("--out", type=str, default=None)
    ap.add_argument("--eval", type=int, default=0, help="held-out parts to evaluate")
    ap.add_argument("--eval-size", type=int, default=192)
    ap.add_argument("--eval-json", type=str, default=None)
    ap.add_argument("--eval-only", action="store_true", help="evaluate the packaged weights, no training")
    ap.add_argument("--max-cg", type=int, default=None, help="iteration cap (default: the reference's 1000)")
    ap.add_argument("--raw-parts", action="store_true",
                    help="evaluate the generated parts as they are, without the reference's island step")
    ap.add_argument("--configs", choices=("headline", "modes", "learned"), default="headline")
    ap.add_argument("--smoothed-level-sweeps", type=int, default=None,
                    help="smoothed_level_sweeps of every configuration (default: the presets')")
    ap.add_argument("--learned-watch", type=int, default=None,
                    help="learned_watch of the configurations with the stage on (default: the option's default)")
    ap.add_argument("--weights", type=str, default=None, help="weights to evaluate (default: the packaged ones)")
    args = ap.parse_args()
    from . import stage
    if args.eval_only:
        params, level = stage.load_weights(args.weights) if args.weights else stage.load_weights()
        seeds = [9_000_000 + 7919 * i for i in range(args.eval)]
        e = args.eval_size
        cfgs = {"headline": headline_configs, "modes": modes_configs,
                "learned": lambda: tuple(c for c in headline_configs() if c[2])}[args.configs]()
        if args.learned_watch is not None:
            for _, opts, use in cfgs:
                if use:
                    opts.learned_watch = int(args.learned_watch)
        if args.smoothed_level_sweeps is not None:
            for _, opts, _ in cfgs:
                opts.smoothed_level_sweeps = int(args.smoothed_level_sweeps)
        rows = evaluate(params, level, seeds, (e, e, e), configs=cfgs, max_cg=args.max_cg,
                        drop_islands=not args.raw_parts)
        _report(rows, cfgs, args)
        return
    sizes = tuple(int(v) for v in args.sizes.split(","))
    snaps = tuple(int(v) for v in args.snapshots.split(","))
    net, hist, secs = train(args.parts, args.level, snaps, args.steps_per_part, lr=args.lr, seed=args.seed,
                            workers=args.workers, sizes=sizes)
    params = net.flat_params()
    if args.out:
        stage.save_weights(args.out, params, args.level, parts=args.parts, snapshots=np.array(snaps),
                           steps=args.parts * args.steps_per_part, seed=args.seed, sizes=np.array(sizes),
                           loss=np.array(hist, dtype=float), train_seconds=secs)
        print(f"[train] saved {args.out} ({params.size} parameters, {secs:.0f}s)")
    if args.eval:
        seeds = [9_000_000 + 7919 * i for i in range(args.eval)]   # disjoint from the training seeds
        e = args.eval_size
        rows = evaluate(params, args.level, seeds, (e, e, e), max_cg=args.max_cg,
                        drop_islands=not args.raw_parts)
        _report(rows, eval_configs(), args)


if __name__ == "__main__":
    main()
