"""The prover steps the reference runs on the CPU, through the oracle: the
permutation products (src/permutation.rs:16-150), the shuffle products
(src/shuffle.rs:16-215) and the multi-open divisions (src/multiopen.rs:145-159,
543-553).  The reference-kernel arm of the proof pipeline
(zkwasm-prover_b200/prover.py with the reference's kernels as symbols) takes
this in place of the library's device entry points, as the reference's own
host does.  Test infrastructure: only the tests and the benchmark's reference
arm use it."""
import numpy as np
import torch

import oracle as O


def _host(t):
    return t.detach().cpu().contiguous().numpy().view(np.uint64).reshape(-1, 4)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()


class OracleHostWork:
    def permutation_products(self, ctx, cols, sigmas, beta, gamma):
        s = ctx.shape
        zs = O.permutation_product([_host(c) for c in cols], [_host(c) for c in sigmas], beta, gamma, ctx.k,
                                   s.chunk_len, ctx.u)
        return [_dev(z) for z in zs]

    def shuffle_products(self, ctx, pairs, beta):
        return [_dev(O.shuffle_product([_host(a)], [_host(b)], beta)) for a, b in pairs]

    def divide_linear(self, ctx, a, z):
        return _dev(O.poly_divide_linear(_host(a), z))
