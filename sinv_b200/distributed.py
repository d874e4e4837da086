"""One process per GPU: sharding the energy loop across ranks.

A transport calculation solves one selected inversion per energy point.  The
points are independent, so they shard across GPUs with no exchange during the
sweeps: every rank takes a cost-balanced share (cost ~ b^3 n per instance),
runs it as one batched launch, and only the quantities that are sums over
energies (the density of states, the gradient dL/dH of an energy-summed loss)
cross ranks, as one all-reduce at the end.  Launch with torchrun, one rank per
GPU, backend ``nccl`` (``gloo`` for CPU tests).
"""

import heapq

import numpy as np


def instance_cost(n, b):
    """Relative cost of one selected inversion: the canonical flop count."""
    return float(b) ** 3 * (9 * n - 8)


def shard_by_cost(costs, world, rank=None):
    """Largest-first greedy partition of instances into ``world`` bins.

    Deterministic (ties broken by index), so every rank computes the same
    plan without communicating.  Returns the index list of ``rank`` or, with
    ``rank=None``, all ranks' lists.
    """
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(world)]
    bins = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        bins[r].append(k)
        heapq.heappush(heap, (load + costs[k], r))
    for b in bins:
        b.sort()
    return bins if rank is None else bins[rank]


def _dist():
    import torch.distributed as dist
    return dist


def rank_and_world(group=None):
    dist = _dist()
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def rgf_batched_sharded(instances, group=None, **kw):
    """Batched RGF of this rank's share of ``instances`` (all ranks pass the
    same list).  Returns ``{index: (G_diag, G_upper, G_lower)}`` for the
    instances this rank computed."""
    from .algorithms.batched import rgf_batched
    rank, world = rank_and_world(group)
    costs = [instance_cost(np.shape(d)[0], np.shape(d)[1]) for d, _, _ in instances]
    mine = shard_by_cost(costs, world, rank)
    if not mine:
        return {}
    out = rgf_batched([instances[k] for k in mine], **kw)
    return dict(zip(mine, out))


def rgf_lesser_batched_sharded(instances, sigmas, group=None, gather=False, compute=None, **kw):
    """Retarded and lesser blocks of this rank's share of the energies: all
    ranks pass the same lists, shares are balanced by cost (largest first) and
    nothing is exchanged during the sweeps.  Returns ``{index: (G_diag,
    G_upper, G_lower, GL_diag, GL_upper, GL_lower)}`` for this rank's
    instances; with ``gather`` every instance's result as host arrays on every
    rank (one ``all_gather_object``).  ``compute`` is the batched call
    (default ``rgf_lesser_batched``; keyword arguments pass through)."""
    if compute is None:
        from .algorithms.lesser import rgf_lesser_batched as compute
    rank, world = rank_and_world(group)
    costs = [instance_cost(np.shape(d)[0], np.shape(d)[1]) for d, _, _ in instances]
    mine = shard_by_cost(costs, world, rank)
    out = dict(zip(mine, compute([instances[k] for k in mine], [sigmas[k] for k in mine], **kw))) if mine else {}
    if not gather or world == 1:
        return out
    host = {k: tuple(np.asarray(x.cpu() if hasattr(x, "cpu") else x) for x in v) for k, v in out.items()}
    parts = [None] * world
    _dist().all_gather_object(parts, host, group=group)
    allres = {}
    for p in parts:
        allres.update(p)
    return allres


def energy_loss_and_grad(H_onsite, H_coupling, energies, eta=1e-3, sigma=0.1, group=None, compute=None):
    """Sum over energies of L(E) = -Im Tr sum_i G_ii(E) / pi and its gradient
    with respect to the Hamiltonian blocks, sharded over ranks.

    ``A(E) = (E + i eta) I - H - Sigma`` with ``Sigma = -i sigma I`` on the
    first and last diagonal blocks; H onsite blocks (n, b, b), couplings
    (n-1, b, b) above the diagonal and their transposes below.  Each rank
    evaluates its share of the energies (``compute(E) -> (loss, g_onsite,
    g_coupling)``, by default the GPU adjoint) and one all-reduce sums the
    loss and both gradients.  Returns ``(loss, g_onsite, g_coupling)`` as torch
    tensors on the inputs' device, identical on every rank.
    """
    import torch
    dist = _dist()
    rank, world = rank_and_world(group)
    n, b = H_onsite.shape[0], H_onsite.shape[1]
    mine = shard_by_cost([1.0] * len(energies), world, rank)
    loss = torch.zeros((), dtype=torch.float64, device=H_onsite.device)
    g_on = torch.zeros_like(H_onsite, dtype=torch.float64)
    g_cp = torch.zeros_like(H_coupling, dtype=torch.float64)
    if compute is None and mine:  # this rank's energies as one batched forward and one batched adjoint
        loss, g_on, g_cp = _gpu_energy_batch(H_onsite, H_coupling, [float(energies[k]) for k in mine], eta, sigma)
    for k in (mine if compute is not None else []):
        l_k, go, gc = compute(float(energies[k]))
        loss += l_k
        g_on += go
        g_cp += gc
    if world > 1:
        flat = torch.cat([loss.reshape(1), g_on.reshape(-1), g_cp.reshape(-1)])
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
        loss = flat[0]
        g_on = flat[1:1 + g_on.numel()].view_as(g_on)
        g_cp = flat[1 + g_on.numel():].view_as(g_cp)
    return loss, g_on, g_cp


def _energy_matrix(Hd, Hu, E, eta, sigma):
    """A(E) = (E + i eta) I - H - Sigma as block arrays (complex128), differentiable in H."""
    import torch
    b = Hd.shape[1]
    eye = torch.eye(b, dtype=torch.complex128, device=Hd.device)
    d = (E + 1j * eta) * eye - Hd.to(torch.complex128)
    edge = torch.zeros_like(d)
    edge[0] = 1j * sigma * eye
    edge[-1] = edge[-1] + 1j * sigma * eye
    return (d + edge, (-Hu.to(torch.complex128)).contiguous(),
            (-Hu.transpose(1, 2).to(torch.complex128)).contiguous())


def _gpu_energy_batch(H_onsite, H_coupling, energies, eta, sigma):
    """Loss and dL/dH over `energies` with one batched forward launch and one
    batched adjoint launch (the energy loop of the gradient as a batch)."""
    import torch
    from .algorithms.adjoint import rgf_batched_autograd
    Hd = H_onsite.detach().clone().requires_grad_(True)
    Hu = H_coupling.detach().clone().requires_grad_(True)
    inst = [_energy_matrix(Hd, Hu, E, eta, sigma) for E in energies]
    out = rgf_batched_autograd(inst)
    loss = sum(-Gd.diagonal(0, 1, 2).imag.sum() / np.pi for (Gd, _, _) in out)
    loss.backward()
    return loss.detach(), Hd.grad.to(torch.float64), Hu.grad.to(torch.float64)


def _gpu_energy_term(H_onsite, H_coupling, eta, sigma):
    import torch
    from .algorithms.adjoint import rgf_autograd

    def term(E):
        Hd = H_onsite.detach().clone().requires_grad_(True)
        Hu = H_coupling.detach().clone().requires_grad_(True)
        b = Hd.shape[1]
        eye = torch.eye(b, dtype=torch.complex128, device=Hd.device)
        d = (E + 1j * eta) * eye - Hd.to(torch.complex128)
        edge = torch.zeros_like(d)
        edge[0] = 1j * sigma * eye
        edge[-1] = edge[-1] + 1j * sigma * eye
        d = d + edge
        u = -Hu.to(torch.complex128)
        l = -Hu.transpose(1, 2).to(torch.complex128)
        Gd, _, _ = rgf_autograd(d, u.contiguous(), l.contiguous())
        loss = -Gd.diagonal(0, 1, 2).imag.sum() / np.pi
        loss.backward()
        return loss.detach(), Hd.grad, Hu.grad

    return term


# --------------------------------------------------------------------------- PSR across ranks
def psr_distributed(local_diag, local_upper, local_lower, n, group=None, gather=False, make_part=None):
    """Parallel Schur reduction of an n-block matrix with rank r of ``group`` as
    partition r, the reference's process layout
    (``src/sinv/algorithms/psr/psr_seqsolve.py:20-73``; at least 3 ranks and 3
    block rows per rank, ``psr_utils.py:55-58``).

    Each rank passes only its partition's block arrays
    (``psr_seqsolve.local_blocks(A_diag, A_upper, A_lower, world, rank)``), so
    a matrix larger than one GPU's memory can be inverted; the reference's
    processes each hold the whole A.  Each rank reduces its partition on its GPU
    (``PsrPart.reduce``); the six boundary slots of every partition cross ranks
    in one ``all_gather`` (the reference's send / recv to rank 0, :313-467);
    every rank solves the small reduced system itself (instead of rank 0
    solving and sending back, :470-645) and produces its partition.  Returns
    this rank's ``(G_diag, G_upper, G_lower)`` in the shapes of its local
    arrays, or with ``gather`` the whole arrays on every rank (the reference
    aggregates on rank 0, :903-943).

    ``make_part`` builds the per-rank compute object (default: ``PsrPart`` on
    the current GPU); it must provide ``reduce()``, ``solve_reduced(Rd, Ru,
    Rl)`` and ``produce(slots, link)``.
    """
    import torch
    from .algorithms import psr_seqsolve as psr
    dist = _dist()
    rank, world = rank_and_world(group)
    part = make_part() if make_part is not None else psr.PsrPart(local_diag, local_upper, local_lower, n, world,
                                                                  rank)
    slots = part.reduce().contiguous()
    if world > 1:
        every = [torch.empty_like(slots) for _ in range(world)]
        dist.all_gather(every, slots, group=group)
    else:
        every = [slots]
    RG = part.solve_reduced(*psr.reduced_system(every, n, world))
    gslots, link = psr.boundary_inverse(RG, rank, world)
    Gd, Gu, Gl = part.produce(gslots, link)
    if not gather:
        return Gd, Gu, Gl
    mmax = psr.part_rows(n, world, 0)[1] + 1  # the first partition is the largest
    buf = torch.zeros((3, mmax) + tuple(Gd.shape[1:]), dtype=Gd.dtype, device=Gd.device)
    buf[0, :Gd.shape[0]] = Gd
    buf[1, :Gu.shape[0]] = Gu
    buf[2, :Gl.shape[0]] = Gl
    pieces = [torch.empty_like(buf) for _ in range(world)] if world > 1 else [buf]
    if world > 1:
        dist.all_gather(pieces, buf, group=group)
    shape = tuple(Gd.shape[1:])
    out = [torch.empty((k,) + shape, dtype=Gd.dtype, device=Gd.device) for k in (n, n - 1, n - 1)]
    for r, pc in enumerate(pieces):
        t, B = psr.part_rows(n, world, r)
        e = min(B + 1, n - 1)
        out[0][t:B + 1] = pc[0, :B + 1 - t]
        out[1][t:e] = pc[1, :e - t]
        out[2][t:e] = pc[2, :e - t]
    return tuple(out)
