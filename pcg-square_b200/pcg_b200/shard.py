"""Combining the partial z of one expansion sharded over ranks.

An expander created with rank/world (pcgb_expander_create_shard) evaluates
only its share of the c(c+1)/2 pair blocks; its z is a partial sum in
[0, p) and the expansion's z is the sum of all ranks' partials mod p
(linearity of z = INTT(sum over pairs)).  Every rank's x is already the
full x.

allreduce_z sums the partials in place, exactly, for any number of ranks:

* up to 4 ranks with the tensor on the GPU: one all-reduce of the words as
  int64 (the two's-complement sum is the uint64 sum, exact since
  4(p - 1) < 2^64), then the library's mod-p pass on the device;
* otherwise: all-gather the partials and add them pairwise mod p, each step
  staying below 2p < 2^63.  For 8 ranks this moves 7N words per rank
  instead of an all-reduce's 1.75N: at N = 2^20, 56 MB, tens of
  microseconds over NVLink beside a 15 ms expansion.
"""
from . import P, reduce_mod_p


def allreduce_z(z, group=None):
    """z: int64 torch tensor of N words in [0, p) (a partial z, viewed as
    int64).  Replaced in place by the sum over the group's ranks mod p."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world == 1:
        return z
    if world <= 4 and z.is_cuda:
        dist.all_reduce(z, group=group)
        st = torch.cuda.current_stream(z.device).cuda_stream
        reduce_mod_p(z.data_ptr(), z.data_ptr(), z.numel(), st)
        return z
    parts = [torch.empty_like(z) for _ in range(world)]
    dist.all_gather(parts, z, group=group)
    acc = parts[0].clone()
    for t in parts[1:]:
        acc += t
        acc -= (acc >= P).to(acc.dtype) * P
    z.copy_(acc)
    return z
