"""Shot sharding over ranks (one process per GPU) and the FWI gradient sum.

Shots are independent until the gradient sum, so each rank runs its own shots
as one batch on its own GPU with no collective on the data path; the only
exchange is the per-iteration sum of the three gradient arrays and the misfit
over ranks, which replaces the reference's element-wise MPI_Allreduce of the
stacked gradient (src/PSV/grad_obj_psv.c:371-390).  Shots go to ranks by
longest-processing-time first on their cost (cells x time steps), so ranks
with uneven shot sizes finish together.

torch.distributed carries the collective: NCCL on GPU tensors in production,
gloo on CPU tensors in the tests.
"""
import numpy as np


def assign_shots(costs, world):
    """LPT assignment: shot indices per rank, each rank's list in shot order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        out[r].append(k)
        load[r] += costs[k]
    return [sorted(x) for x in out]


def allreduce_sum(arrays, dist=None, device=None):
    """Sums float arrays over all ranks (in float64) and returns them on the host.
    dist: torch.distributed (initialised) or None for a single process."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [np.asarray(a, np.float64) for a in arrays]
    import torch

    flat = np.concatenate([np.asarray(a, np.float64).ravel() for a in arrays])
    t = torch.from_numpy(flat)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    flat = t.cpu().numpy()
    out, o = [], 0
    for a in arrays:
        n = np.asarray(a).size
        out.append(flat[o:o + n].reshape(np.shape(a)))
        o += n
    return out


def make_shot(model, sh):
    """A Shot from a shot tuple (src_i, src_j, signals, rec_i, rec_j[, src_type[, src_azi[, (x, z)]]])."""
    from . import api as dn

    return dn.Shot(model, *sh[:5], src_type=sh[5] if len(sh) > 5 else None, src_azi=sh[6] if len(sh) > 6 else None)


def source_position(sh, dh):
    """The shot's first source in metres: the table's (x, z) when the tuple carries
    it (as the reference's srcpos), else its grid cell times DH."""
    if len(sh) > 7 and sh[7] is not None:
        return float(sh[7][0]), float(sh[7][1])
    return float(sh[0][0]) * dh, float(sh[1][0]) * dh


def memory_batches(params, shots, idx, store, device=0, share=0.9):
    """idx split into batches that fit `share` of the device's free memory (the
    library's cached blocks counted as free), spread evenly: 32 shots that fit
    9 at a time run as 4 x 8."""
    from . import api as dn

    idx = list(idx)
    if not idx:
        return []
    ntr = max(len(shots[k][3]) for k in idx)
    fp = dn.shot_footprint(params, ntr, store)
    free, _ = dn.device_memory(device)
    most = max(1, int(share * free / max(fp, 1)))
    nb = -(-len(idx) // most)
    size = -(-len(idx) // nb)
    return [idx[k:k + size] for k in range(0, len(idx), size)]


def sharded_gradient(params, model, shots, obs, dist=None, device_index=0, shot_taper=None, residual=None,
                     energy=None, misfit_shots=None):
    """FWI gradient of `shots` sharded over the ranks of `dist` (all ranks pass
    the same arguments).  Each rank runs its share in batches that fit its GPU's memory:
    forward with snapshots, device residuals against `obs`, adjoint, and stacks
    its shots' gradients in shot order; the partial gradients and misfits are
    then summed over ranks.  Returns (g_vp, g_vs, g_rho, misfit), float64, on
    every rank.  shot_taper = (srtshape, srtradius, filtsize) applies the
    per-shot circular taper (taper_grad_shot.c) around each shot's first source
    before stacking; residual = the calc_res options of Shot.residual_ex (LNORM,
    N_ORDER, OFFSET_MUTE, ...; None: the L2 residual); energy = (C_vp, C_vs,
    C_rho) scales each shot's gradient by its energy weights (EPRECOND 1 or 3
    in params); misfit_shots: the indices whose misfit is summed (the reference's
    test shots, TESTSHOT_START..END by INCR; None: all)."""
    from . import api as dn
    from ._lib import MODE_ADJOINT, MODE_FORWARD, SEC_VX, SEC_VY

    rank = dist.get_rank() if dist is not None and dist.is_initialized() else 0
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    costs = [params.nx * params.ny * params.nt for _ in shots]
    mine = assign_shots(costs, world)[rank]
    g = [np.zeros((params.nx, params.ny), np.float64) for _ in range(3)]
    misfit = 0.0
    if mine:
        m = dn.Model(params, *model[:3], model[3] if params.L else None, model[4] if params.L else None,
                     device=device_index)
        for part in memory_batches(params, shots, mine, 1, device_index):
            ss = [make_shot(m, shots[k]) for k in part]
            dn.run(ss, MODE_FORWARD)
            for s, k in zip(ss, part):
                if residual is None:
                    mk = s.residual(obs[k][0], SEC_VX) + s.residual(obs[k][1], SEC_VY)
                else:
                    sx, sz = source_position(shots[k], params.dh)
                    opts = dict({"src_x": sx, "src_z": sz}, **residual)
                    mk = s.residual_ex(obs[k][0], SEC_VX, **opts) + s.residual_ex(obs[k][1], SEC_VY, **opts)
                if misfit_shots is None or k in misfit_shots:
                    misfit += mk
            dn.run(ss, MODE_ADJOINT)
            for s, k in zip(ss, part):   # stacked in shot order, batch after batch
                if shot_taper is None and energy is None:
                    s.accumulate_gradient()
                else:
                    sx, sz = source_position(shots[k], params.dh)
                    s.accumulate_gradient_ex(energy=energy, circular_taper=None if shot_taper is None
                                             else tuple(shot_taper) + (sx, sz))
            for s in ss:
                s.close()
        g = [x.astype(np.float64) for x in m.gradient()]
        m.close()
    dev = None
    if dist is not None and dist.is_initialized() and dist.get_backend() == "nccl":
        dev = f"cuda:{device_index}"
    red = allreduce_sum(g + [np.array([misfit])], dist, dev)
    return red[0], red[1], red[2], float(red[3][0])
