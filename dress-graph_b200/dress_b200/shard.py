"""Delta^k / Nabla^k sharded over processes, one per GPU.

The reference's MPI layer (libdress/src/mpi/dress_mpi.c:43-145) gives rank r
of P the subsets with lexicographic rank s = r (mod P) -- the strided call
with offset = r, stride = P -- then gathers every rank's flat histogram and
merges them.  Here each rank runs its stride through the batched engine on
its own GPU, the flat histograms cross once through ``torch.distributed``
(NCCL between GPUs, gloo on CPUs) and ``dressx_hist_merge`` merges them.
There is no exchange during the fits.
"""
import ctypes

import numpy as np

from . import _abi


def merge_hists(flats):
    """Merge flat int64 [value_bits, count, ...] lists (each ascending by
    value) of disjoint shards into one list of the same form."""
    lib = _abi.load()
    arrs = [np.ascontiguousarray(f, dtype=np.int64) for f in flats]
    n = len(arrs)
    ptrs = (ctypes.POINTER(ctypes.c_int64) * max(1, n))()
    lens = (ctypes.c_int64 * max(1, n))()
    for i, a in enumerate(arrs):
        ptrs[i] = a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        lens[i] = a.size
    out = ctypes.POINTER(ctypes.c_int64)()
    out_len = ctypes.c_int64()
    code = lib.dressx_hist_merge(ptrs, lens, n, ctypes.byref(out), ctypes.byref(out_len))
    if code != 0:
        raise RuntimeError(f"dressx_hist_merge failed ({code}): {_abi.last_error()[1]}")
    if out_len.value == 0:
        return np.zeros(0, dtype=np.int64)
    res = np.ctypeslib.as_array(out, shape=(out_len.value,)).copy()
    lib.dressx_free(ctypes.cast(out, ctypes.c_void_p))
    return res


def gather_hists(local, group=None):
    """All-gather variable-length flat histograms: every rank gets the list
    of all ranks' arrays (rank order)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(local, dtype=np.int64)).to(dev)
    size = torch.tensor([t.numel()], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(size) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    sizes = [int(s.item()) for s in sizes]
    top = max(sizes) if sizes else 0
    pad = torch.zeros(top, dtype=torch.int64, device=dev)
    pad[: t.numel()] = t
    bufs = [torch.zeros(top, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return [b[:s].cpu().numpy() for b, s in zip(bufs, sizes)]


def fit_sharded(graph, kind=0, k=1, group=None, max_iterations=100, epsilon=1e-6, n_samples=0, seed=0):
    """This rank's stride of a Delta^k (kind 0) or Nabla^k (kind 1) request on
    its GPU, then the merged histogram of all ranks.  Returns (flat,
    num_subgraphs, fits of all ranks)."""
    import torch
    import torch.distributed as dist
    from . import hist_requests
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    flat, _, nsub, fits, status = hist_requests([graph], kind, k, max_iterations=max_iterations, epsilon=epsilon,
                                                n_samples=n_samples, seed=seed, offset=rank, stride=world)[0]
    if status != 0:
        raise RuntimeError(f"rank {rank}: request failed with status {status}")
    merged = merge_hists(gather_hists(flat, group))
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    f = torch.tensor([fits], dtype=torch.int64, device=dev)
    dist.all_reduce(f, group=group)
    return merged, nsub, int(f.item())
