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


def _world(dist):
    if dist is None or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


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


def allreduce_scalar(x, dist=None, device=None):
    """The sum of a float over all ranks (float64)."""
    return float(allreduce_sum([np.array([x])], dist, device)[0][0])


def allreduce_model_gradient(model, dist=None):
    """Sums a model's stacked gradients over the ranks of `dist` in place, in
    float64 on the device: the gradients are exported into a device tensor
    (dn_model_gradient_to_device), all-reduced (NCCL on the device; gloo through
    a host copy of that tensor) and imported back.  This replaces the
    reference's element-wise MPI_Allreduce of the stacked gradient
    (src/PSV/grad_obj_psv.c:371-390).  A single process does nothing."""
    rank, world = _world(dist)
    if world == 1:
        return
    import torch

    from ._lib import check, lib

    p = model.params
    dev = torch.device(f"cuda:{model.device}")
    t = torch.empty(3 * p.nx * p.ny, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    check(lib.dn_model_gradient_to_device(model.handle, t.data_ptr()))
    if dist.get_backend() == "nccl":
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    else:
        h = t.cpu()
        dist.all_reduce(h, op=dist.ReduceOp.SUM)
        t.copy_(h)
    torch.cuda.synchronize(dev)
    check(lib.dn_model_gradient_from_device(model.handle, t.data_ptr()))


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
    9 at a time run as 4 x 8.  A shot larger than the free memory raises
    MemoryError before any batch runs."""
    from . import api as dn

    idx = list(idx)
    if not idx:
        return []
    ntr = max(len(shots[k][3]) for k in idx)
    fp = dn.shot_footprint(params, ntr, store)
    free, _ = dn.device_memory(device)
    if fp > free:
        raise MemoryError(f"one shot needs {fp} bytes of device memory and {free} are free on device {device}")
    most = max(1, int(share * free / max(fp, 1)))
    nb = -(-len(idx) // most)
    size = -(-len(idx) // nb)
    return [idx[k:k + size] for k in range(0, len(idx), size)]


def shard_of(params, idx, dist=None):
    """This rank's share of the shot indices idx (LPT over equal costs: round robin)."""
    rank, world = _world(dist)
    idx = list(idx)
    costs = [params.nx * params.ny * params.nt for _ in idx]
    return [idx[k] for k in assign_shots(costs, world)[rank]]


def gradient_model(params, model, shots, obs, dist=None, device_index=0, shot_taper=None, residual=None,
                   energy=None, misfit_shots=None):
    """FWI gradient of `shots` sharded over the ranks of `dist` (all ranks pass
    the same arguments), kept on the device.  Each rank runs its share in
    batches that fit its GPU's memory: forward with snapshots, device residuals
    against `obs`, adjoint, and stacks its shots' gradients in shot order into a
    Model of `model`; the stacked gradients are then summed over ranks on the
    device (allreduce_model_gradient) and the misfits as one scalar.  Returns
    (Model, misfit): the Model holds the summed gradients (Model.gradient() reads
    them) and is the caller's to close.

    shot_taper = (srtshape, srtradius, filtsize) applies the per-shot circular
    taper (taper_grad_shot.c) around each shot's first source before stacking;
    residual = the calc_res options of Shot.residual_ex (LNORM, N_ORDER,
    OFFSET_MUTE, ...; None: the L2 residual); energy = (C_vp, C_vs, C_rho)
    scales each shot's gradient by its energy weights (EPRECOND 1 or 3 in
    params); misfit_shots: the indices whose misfit is summed (the reference's
    test shots, TESTSHOT_START..END by INCR; None: all)."""
    from . import api as dn
    from ._lib import MODE_ADJOINT, MODE_FORWARD, SEC_VX, SEC_VY

    mine = shard_of(params, range(len(shots)), dist)
    misfit = 0.0
    m = dn.Model(params, *model[:3], model[3] if params.L else None, model[4] if params.L else None,
                 device=device_index)
    try:
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
        allreduce_model_gradient(m, dist)
        misfit = allreduce_scalar(misfit, dist, _collective_device(dist, device_index))
    except BaseException:
        m.close()
        raise
    return m, misfit


def _collective_device(dist, device_index):
    if dist is not None and dist.is_initialized() and dist.get_backend() == "nccl":
        return f"cuda:{device_index}"
    return None


def sharded_gradient(params, model, shots, obs, dist=None, device_index=0, shot_taper=None, residual=None,
                     energy=None, misfit_shots=None):
    """gradient_model's gradients fetched to the host: (g_vp, g_vs, g_rho,
    misfit), float64 arrays in file order, on every rank."""
    m, misfit = gradient_model(params, model, shots, obs, dist, device_index, shot_taper, residual, energy,
                               misfit_shots)
    g = [x.astype(np.float64) for x in m.gradient()]
    m.close()
    return g[0], g[1], g[2], misfit


def sharded_misfit(params, model, shots, obs, idx, dist=None, device_index=0, residual=None):
    """The objective of obj_psv.c: mode-2 forward runs of the shots idx on
    `model`, each rank running its share (src/PSV/obj_psv.c:48 loops over its
    own shots) in batches that fit its GPU, the vx and vy misfits summed over
    the rank's shots and then over ranks as one scalar (obj_psv.c:233)."""
    from . import api as dn
    from ._lib import MODE_OBJECTIVE, SEC_VX, SEC_VY

    p = params.replace(store_snapshots=0, ckpt_steps=0)
    mine = shard_of(p, idx, dist)
    L2 = 0.0
    if mine:
        m = dn.Model(p, *model[:3], model[3] if p.L else None, model[4] if p.L else None, device=device_index)
        try:
            for part in memory_batches(p, shots, mine, 0, device_index):
                ss = [make_shot(m, shots[k]) for k in part]
                dn.run(ss, MODE_OBJECTIVE)
                for s, k in zip(ss, part):
                    ovx, ovy = obs[k]
                    if residual is None:
                        L2 += s.residual(ovx, SEC_VX) + s.residual(ovy, SEC_VY)
                    else:
                        sx, sz = source_position(shots[k], p.dh)
                        opts = dict({"src_x": sx, "src_z": sz}, **residual)
                        L2 += s.residual_ex(ovx, SEC_VX, **opts) + s.residual_ex(ovy, SEC_VY, **opts)
                for s in ss:
                    s.close()
        finally:
            m.close()
    return allreduce_scalar(L2, dist, _collective_device(dist, device_index))
