// Elementwise kernels of the quotient (eval_h) evaluation on the extended
// domain, one thread per row, grid-stride, rotations taken modulo n.
//
// Reference kernels restated (cuda/bn254.cu): _field_op 585-639,
// _field_op_batch_mul_sum 542-572, _extended_prepare 641-662,
// _permutation_eval_h_p1/p2/l 664-765, _lookup_eval_h 798-865,
// _logup_eval_h 867-921, _logup_eval_h_extra_inputs 924-948,
// _shuffle_eval_h 975-1015, _shuffle_eval_h_v2 1017-1071, _field_mul_zip
// 1121-1131, _field_sum 496-540, _shplonk_h_x_merge 1133-1149,
// _logup_eval_h_inputs_product_sum 1172-1213.  The formulas are the same
// polynomial identities; the launch shapes are not (the reference uses
// 64-thread blocks and requires n to be a multiple of 64).
#include "common.cuh"
#include "kernels.h"

namespace zk {

static __device__ __forceinline__ uint32_t rot_idx(uint32_t i, int rot, uint32_t n) {
    // (i + rot) mod n for any sign of rot; n need not be a power of two
    long long r = ((long long)i + rot) % (long long)n;
    if (r < 0) r += n;
    return (uint32_t)r;
}

static __device__ __forceinline__ uint32_t rot_pow2(uint32_t i, int rot, uint32_t n) {
    return (uint32_t)((int)i + rot) & (n - 1);
}

#define ZK_GRID_LOOP(i, n) \
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

static inline unsigned grid_for(uint32_t n, unsigned tb = 256) {
    uint64_t b = ((uint64_t)n + tb - 1) / tb;
    if (b > 148u * 32u) b = 148u * 32u;
    if (b == 0) b = 1;
    return (unsigned)b;
}

// ------------------------------------------------------------------ field_op

// a column times its constant is a product by a known factor; operands stay
// lazily reduced until the store
__global__ void field_op_kernel(Fr* res, const Fr* l, int l_rot, const Fr* l_c, const Fr* r, int r_rot,
                                const Fr* r_c, uint32_t n, int op) {
    __shared__ KnownFr kl, kr;
    if (threadIdx.x == 0) {
        if (l && l_c) kl = known_fr(ld_elem<FrCfg>(l_c));
        if (r && r_c) kr = known_fr(ld_elem<FrCfg>(r_c));
    }
    __syncthreads();
    ZK_GRID_LOOP(i, n) {
        Fr fl, fr_;
        if (l) {
            fl = ld_elem<FrCfg>(l + rot_idx(i, l_rot, n));
            if (l_c) fl = mul_known(fl, kl);
        } else {
            fl = ld_elem<FrCfg>(l_c);
        }
        if (r) {
            fr_ = ld_elem<FrCfg>(r + rot_idx(i, r_rot, n));
            if (r_c) fr_ = mul_known(fr_, kr);
        } else if (r_c) {
            fr_ = ld_elem<FrCfg>(r_c);
        } else {
            fr_ = fe_zero<FrCfg>();
        }
        Fr out;
        if (op == 0)
            out = fe_canon<FrCfg>(fe_add_lazy<FrCfg>(fl, fr_));
        else if (op == 1)
            out = fe_mul<FrCfg>(fl, fr_);
        else if (op == 2)
            out = fe_canon<FrCfg>(fl);
        else
            out = fe_canon<FrCfg>(fe_sub_lazy<FrCfg>(fl, fr_));
        st_elem<FrCfg>(res + i, out);
    }
}

cudaError_t field_op(Fr* res, const Fr* l, int l_rot, const Fr* l_c, const Fr* r, int r_rot, const Fr* r_c,
                     uint32_t n, int op, cudaStream_t s) {
    if (op < 0 || op > 3) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    if (!l && !l_c) return cudaErrorInvalidValue;
    // the rows are read rotated, so an in-place rotated operand needs a
    // snapshot; the reference has the same hazard and callers avoid it
    field_op_kernel<<<grid_for(n), 256, 0, s>>>(res, l, l_rot, l_c, r, r_rot, r_c, n, op);
    return cudaGetLastError();
}

// --------------------------------------------------- field_op_batch_mul_sum
// v = [coeff0, a00, a01, .., null, coeff1, a10, .., null, ...] (device array of
// device pointers), rot = rotation per non-coefficient entry.

// The term list (pointers and rotations) is staged in shared memory once per
// block when it fits (every row walks it), together with each term's
// coefficient in the pair form of a known factor, so that a term's first
// product (coefficient x first column) is a product by a known factor.  Each
// term's product is kept lazily reduced in [0, 2r) until the row's sum is
// stored.
static constexpr int BMS_SMEM_ENTRIES = 256;
// a term takes at least two entries (its coefficient and its null)
static constexpr int BMS_SMEM_TERMS = BMS_SMEM_ENTRIES / 2;

__global__ void batch_mul_sum_kernel(Fr* res, Fr* const* v, const int* rot, int n_v, uint32_t n) {
    __shared__ const Fr* sv[BMS_SMEM_ENTRIES];
    __shared__ int srot[BMS_SMEM_ENTRIES];
    __shared__ KnownFr scoef[BMS_SMEM_TERMS];
    if (n_v <= BMS_SMEM_ENTRIES) {
        for (int k = threadIdx.x; k < n_v; k += blockDim.x) sv[k] = v[k];
        __syncthreads();
        // rotations are indexed by the non-null, non-coefficient entries (at
        // most n_v of them); term k's coefficient pair is built by thread k
        int nrot = 0, nterm = 0;
        {
            int vi = 0;
            while (vi < n_v) {
                if (nterm == (int)threadIdx.x) scoef[nterm] = known_fr(ld_elem<FrCfg>(sv[vi]));
                vi++;
                while (vi < n_v && sv[vi]) {
                    vi++;
                    nrot++;
                }
                vi++;
                nterm++;
            }
        }
        for (int k = threadIdx.x; k < nrot; k += blockDim.x) srot[k] = rot[k];
        __syncthreads();
        ZK_GRID_LOOP(i, n) {
            Fr acc = fe_zero<FrCfg>();
            int vi = 0, ri = 0, tk = 0;
            while (vi < n_v) {
                Fr t;
                if (vi + 1 < n_v && sv[vi + 1]) {
                    t = mul_known(ld_elem<FrCfg>(sv[vi + 1] + rot_pow2(i, srot[ri], n)), scoef[tk]);
                    vi += 2;
                    ri++;
                } else {
                    t = ld_elem<FrCfg>(sv[vi++]);  // a term without columns
                }
                while (vi < n_v && sv[vi]) {
                    t = fe_mul_lazy<FrCfg>(t, ld_elem<FrCfg>(sv[vi] + rot_pow2(i, srot[ri], n)));
                    vi++;
                    ri++;
                }
                acc = fe_add_lazy<FrCfg>(acc, t);
                vi++;
                tk++;
            }
            st_elem<FrCfg>(res + i, fe_add<FrCfg>(ld_elem<FrCfg>(res + i), fe_canon<FrCfg>(acc)));
        }
        return;
    }
    ZK_GRID_LOOP(i, n) {
        Fr acc = fe_zero<FrCfg>();
        int vi = 0, ri = 0;
        while (vi < n_v) {
            Fr t = ld_elem<FrCfg>(v[vi++]);
            while (vi < n_v && v[vi]) {
                t = fe_mul_lazy<FrCfg>(t, ld_elem<FrCfg>(v[vi] + rot_pow2(i, rot[ri], n)));
                vi++;
                ri++;
            }
            acc = fe_add_lazy<FrCfg>(acc, t);
            vi++;
        }
        st_elem<FrCfg>(res + i, fe_add<FrCfg>(ld_elem<FrCfg>(res + i), fe_canon<FrCfg>(acc)));
    }
}

cudaError_t field_op_batch_mul_sum(Fr* res, Fr* const* v, const int* rot, int n_v, uint32_t n, cudaStream_t s) {
    if (n == 0 || n_v <= 0) return cudaSuccess;
    batch_mul_sum_kernel<<<grid_for(n), 256, 0, s>>>(res, v, rot, n_v, n);
    return cudaGetLastError();
}

// ----------------------------------------------------------- extended_prepare

__global__ void extended_prepare_kernel(Fr* s, const Fr* cp, uint32_t cpn, uint32_t n) {
    ZK_GRID_LOOP(i, n) {
        uint32_t k = i % cpn;
        if (k != 0) st_elem<FrCfg>(s + i, fe_mul<FrCfg>(ld_elem<FrCfg>(s + i), ld_elem<FrCfg>(cp + k - 1)));
    }
}

cudaError_t extended_prepare(Fr* s, const Fr* coset_powers, uint32_t cpn, uint32_t size, uint32_t ext_size,
                             int to_coset, cudaStream_t st) {
    if (cpn == 0) return cudaErrorInvalidValue;
    uint32_t lim = size;
    if (to_coset) {
        lim = ext_size;
    } else if (ext_size > size) {
        ZK_CHECK(cudaMemsetAsync(s + size, 0, (size_t)(ext_size - size) * sizeof(Fr), st));
    }
    if (lim == 0 || cpn == 1) return cudaGetLastError();
    extended_prepare_kernel<<<grid_for(lim), 256, 0, st>>>(s, coset_powers, cpn, lim);
    return cudaGetLastError();
}

// --------------------------------------------------------------- permutation

__global__ void perm_p1_kernel(Fr* res, const Fr* first, const Fr* last, const Fr* l0, const Fr* l_last,
                               const Fr* y, uint32_t n) {
    const KnownFr ky = block_known(y);
    const Fr one = fe_one<FrCfg>();
    ZK_GRID_LOOP(i, n) {
        Fr t1 = mul_known(ld_elem<FrCfg>(res + i), ky);
        Fr t2 = fe_mul_lazy<FrCfg>(fe_sub_lazy<FrCfg>(one, ld_elem<FrCfg>(first + i)), ld_elem<FrCfg>(l0 + i));
        t1 = mul_known(fe_add_lazy<FrCfg>(t1, t2), ky);
        Fr z = ld_elem<FrCfg>(last + i);
        t2 = fe_mul_lazy<FrCfg>(fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(z, z), z), ld_elem<FrCfg>(l_last + i));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(fe_add_lazy<FrCfg>(t1, t2)));
    }
}

cudaError_t permutation_eval_h_p1(Fr* res, const Fr* first_set, const Fr* last_set, const Fr* l0,
                                  const Fr* l_last, const Fr* y, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    perm_p1_kernel<<<grid_for(n), 256, 0, s>>>(res, first_set, last_set, l0, l_last, y, n);
    return cudaGetLastError();
}

// The reference's chain t = t y + (set_j[i] - set_{j-1}[i + rot]) l0 over
// j = 1 .. k-1 (k = n_set) equals res y^(k-1) + l0 u with
// u = sum_j y^(k-1-j) (set_j[i] - set_{j-1}[i + rot]) by Horner: k - 1 products
// by the known factors y and y^(k-1) and one by l0, instead of k - 1 of each.
__global__ void __launch_bounds__(256, 4) perm_p2_kernel(Fr* res, const Fr* const* set, const Fr* l0, const Fr* y,
                                                          int n_set, int rot, uint32_t n) {
    __shared__ KnownFr sk[2];
    if (threadIdx.x == 0) {
        const Fr yy = ld_elem<FrCfg>(y);
        Fr yk = yy;
        for (int j = 2; j < n_set; j++) yk = fe_mul<FrCfg>(yk, yy);
        sk[0] = known_fr(yy);
        sk[1] = known_fr(yk);
    }
    __syncthreads();
    const KnownFr &ky = sk[0], &kyk = sk[1];
    ZK_GRID_LOOP(i, n) {
        const uint32_t rp = rot_pow2(i, rot, n);
        // lazily reduced in [0, 2r) until the store
        Fr u = fe_sub_lazy<FrCfg>(ld_elem<FrCfg>(set[1] + i), ld_elem<FrCfg>(set[0] + rp));
        for (int j = 2; j < n_set; j++)
            u = fe_add_lazy<FrCfg>(mul_known(u, ky),
                                   fe_sub_lazy<FrCfg>(ld_elem<FrCfg>(set[j] + i), ld_elem<FrCfg>(set[j - 1] + rp)));
        const Fr t = fe_add_lazy<FrCfg>(mul_known(ld_elem<FrCfg>(res + i), kyk),
                                        fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(l0 + i)));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(t));
    }
}

cudaError_t permutation_eval_h_p2(Fr* res, const Fr* const* set, const Fr* l0, const Fr* y, int n_set, int rot,
                                  uint32_t n, cudaStream_t s) {
    if (n == 0 || n_set < 2) return cudaSuccess;
    perm_p2_kernel<<<grid_for(n), 256, 0, s>>>(res, set, l0, y, n_set, rot, n);
    return cudaGetLastError();
}

__global__ void perm_l_kernel(Fr* res, const Fr* beta, const Fr* gamma, const Fr* p, uint32_t n) {
    const KnownFr kb = block_known(beta);
    ZK_GRID_LOOP(i, n) {
        Fr t = mul_known(ld_elem<FrCfg>(p + i), kb);
        if (i == 0) t = fe_add_lazy<FrCfg>(t, ld_elem<FrCfg>(gamma));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(fe_add_lazy<FrCfg>(ld_elem<FrCfg>(res + i), t)));
    }
}

cudaError_t permutation_eval_h_l(Fr* res, const Fr* beta, const Fr* gamma, const Fr* p, uint32_t n,
                                 cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    perm_l_kernel<<<grid_for(n), 256, 0, s>>>(res, beta, gamma, p, n);
    return cudaGetLastError();
}

// --------------------------------------------------------------------- lookup

__global__ void lookup_kernel(Fr* res, const Fr* input, const Fr* table, const Fr* pin, const Fr* ptab,
                              const Fr* z, const Fr* l0, const Fr* l_last, const Fr* l_act, const Fr* y,
                              const Fr* beta, const Fr* gamma, int rot, uint32_t n) {
    const KnownFr ky = block_known(y);
    const Fr bb = ld_elem<FrCfg>(beta), gg = ld_elem<FrCfg>(gamma);
    const Fr one = fe_one<FrCfg>();
    ZK_GRID_LOOP(i, n) {
        const uint32_t rn = rot_pow2(i, rot, n), rp = rot_pow2(i, -rot, n);
        const Fr zi = ld_elem<FrCfg>(z + i);
        Fr t = mul_known(ld_elem<FrCfg>(res + i), ky);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(l0 + i), fe_sub_lazy<FrCfg>(one, zi)));
        t = mul_known(t, ky);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(l_last + i),
                                                     fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(zi, zi), zi)));
        t = mul_known(t, ky);
        const Fr a = ld_elem<FrCfg>(pin + i), sv = ld_elem<FrCfg>(ptab + i);
        Fr u = fe_mul_lazy<FrCfg>(fe_add_lazy<FrCfg>(a, bb), fe_add_lazy<FrCfg>(sv, gg));
        u = fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(z + rn));
        Fr x = fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(input + i), ld_elem<FrCfg>(table + i));
        u = fe_sub_lazy<FrCfg>(u, fe_mul_lazy<FrCfg>(zi, x));
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(l_act + i)));
        t = mul_known(t, ky);
        const Fr p = fe_sub_lazy<FrCfg>(a, sv);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(l0 + i), p));
        t = mul_known(t, ky);
        u = fe_mul_lazy<FrCfg>(fe_sub_lazy<FrCfg>(a, ld_elem<FrCfg>(pin + rp)), p);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(l_act + i)));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(t));
    }
}

cudaError_t lookup_eval_h(Fr* res, const Fr* input, const Fr* table, const Fr* permuted_input,
                          const Fr* permuted_table, const Fr* z, const Fr* l0, const Fr* l_last,
                          const Fr* l_active_row, const Fr* y, const Fr* beta, const Fr* gamma, int rot, uint32_t n,
                          cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    lookup_kernel<<<grid_for(n), 256, 0, s>>>(res, input, table, permuted_input, permuted_table, z, l0, l_last,
                                              l_active_row, y, beta, gamma, rot, n);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------- logup

__global__ void logup_kernel(Fr* res, const Fr* ip, const Fr* ips, const Fr* table, const Fr* m, const Fr* zf,
                             const Fr* zl, const Fr* l0, const Fr* l_last, const Fr* l_act, const Fr* y, int rot,
                             uint32_t n) {
    const KnownFr ky = block_known(y);
    ZK_GRID_LOOP(i, n) {
        const uint32_t rn = rot_pow2(i, rot, n);
        const Fr z = ld_elem<FrCfg>(zf + i);
        Fr t = mul_known(ld_elem<FrCfg>(res + i), ky);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(l0 + i), z));
        t = mul_known(t, ky);
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(l_last + i), ld_elem<FrCfg>(zl + i)));
        t = mul_known(t, ky);
        const Fr tab = ld_elem<FrCfg>(table + i);
        Fr u = fe_mul_lazy<FrCfg>(fe_sub_lazy<FrCfg>(ld_elem<FrCfg>(zf + rn), z), tab);
        u = fe_add_lazy<FrCfg>(u, ld_elem<FrCfg>(m + i));
        u = fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(ip + i));
        u = fe_sub_lazy<FrCfg>(u, fe_mul_lazy<FrCfg>(tab, ld_elem<FrCfg>(ips + i)));
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(l_act + i)));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(t));
    }
}

cudaError_t logup_eval_h(Fr* res, const Fr* input_product, const Fr* input_product_sum, const Fr* table,
                         const Fr* multiplicity, const Fr* z_first, const Fr* z_last, const Fr* l0,
                         const Fr* l_last, const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    logup_kernel<<<grid_for(n), 256, 0, s>>>(res, input_product, input_product_sum, table, multiplicity, z_first,
                                             z_last, l0, l_last, l_active_row, y, rot, n);
    return cudaGetLastError();
}

__global__ void logup_extra_kernel(Fr* res, const Fr* ip, const Fr* ips, const Fr* z, const Fr* l_act,
                                   const Fr* y, int rot, uint32_t n) {
    const KnownFr ky = block_known(y);
    ZK_GRID_LOOP(i, n) {
        const uint32_t rn = rot_pow2(i, rot, n);
        Fr t = mul_known(ld_elem<FrCfg>(res + i), ky);
        Fr u = fe_sub_lazy<FrCfg>(ld_elem<FrCfg>(z + rn), ld_elem<FrCfg>(z + i));
        u = fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(ip + i));
        u = fe_sub_lazy<FrCfg>(u, ld_elem<FrCfg>(ips + i));
        t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(u, ld_elem<FrCfg>(l_act + i)));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(t));
    }
}

cudaError_t logup_eval_h_extra_inputs(Fr* res, const Fr* input_product, const Fr* input_product_sum, const Fr* z,
                                      const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    logup_extra_kernel<<<grid_for(n), 256, 0, s>>>(res, input_product, input_product_sum, z, l_active_row, y, rot,
                                                   n);
    return cudaGetLastError();
}

__global__ void inputs_product_sum_kernel(Fr* prod, Fr* psum, const Fr* const* set, int n_set, uint32_t n) {
    ZK_GRID_LOOP(i, n) {
        // prefix and suffix products give every leave-one-out product in 3k mults
        Fr p = fe_one<FrCfg>();
        Fr sum = fe_zero<FrCfg>();
        // running: sum_{j<k} prod_{l<=k, l!=j} a_l  updated as sum = sum * a_k + p_{k-1}
        for (int k = 0; k < n_set; k++) {
            const Fr a = ld_elem<FrCfg>(set[k] + i);
            sum = fe_add_lazy<FrCfg>(fe_mul_lazy<FrCfg>(sum, a), p);
            p = fe_mul_lazy<FrCfg>(p, a);
        }
        st_elem<FrCfg>(prod + i, fe_canon<FrCfg>(p));
        st_elem<FrCfg>(psum + i, fe_canon<FrCfg>(sum));
    }
}

cudaError_t logup_eval_h_inputs_product_sum(Fr* product, Fr* product_sum, const Fr* const* set, int n_set,
                                            uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    inputs_product_sum_kernel<<<grid_for(n), 256, 0, s>>>(product, product_sum, set, n_set, n);
    return cudaGetLastError();
}

// -------------------------------------------------------------------- shuffle

// lhs, rhs lazily reduced; the result canonical
__device__ __forceinline__ Fr shuffle_tail(Fr t, const KnownFr& ky, const Fr& zi, const Fr& zn, const Fr& l0,
                                           const Fr& ll, const Fr& la, const Fr& lhs, const Fr& rhs) {
    const Fr one = fe_one<FrCfg>();
    t = mul_known(t, ky);
    t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(l0, fe_sub_lazy<FrCfg>(one, zi)));
    t = mul_known(t, ky);
    t = fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(ll, fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(zi, zi), zi)));
    t = mul_known(t, ky);
    Fr u = fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(rhs, zn), fe_mul_lazy<FrCfg>(lhs, zi));
    return fe_canon<FrCfg>(fe_add_lazy<FrCfg>(t, fe_mul_lazy<FrCfg>(u, la)));
}

__global__ void shuffle_kernel(Fr* res, const Fr* input, const Fr* table, const Fr* z, const Fr* l0,
                               const Fr* l_last, const Fr* l_act, const Fr* y, int rot, uint32_t n) {
    const KnownFr ky = block_known(y);
    ZK_GRID_LOOP(i, n) {
        const uint32_t rn = rot_pow2(i, rot, n);
        Fr t = shuffle_tail(ld_elem<FrCfg>(res + i), ky, ld_elem<FrCfg>(z + i), ld_elem<FrCfg>(z + rn),
                            ld_elem<FrCfg>(l0 + i), ld_elem<FrCfg>(l_last + i), ld_elem<FrCfg>(l_act + i),
                            ld_elem<FrCfg>(input + i), ld_elem<FrCfg>(table + i));
        st_elem<FrCfg>(res + i, t);
    }
}

cudaError_t shuffle_eval_h(Fr* res, const Fr* input, const Fr* table, const Fr* z, const Fr* l0, const Fr* l_last,
                           const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    shuffle_kernel<<<grid_for(n), 256, 0, s>>>(res, input, table, z, l0, l_last, l_active_row, y, rot, n);
    return cudaGetLastError();
}

__global__ void shuffle_v2_kernel(Fr* res, const Fr* const* inputs, const Fr* const* tables, const Fr* betas,
                                  int group_len, const Fr* z, const Fr* l0, const Fr* l_last, const Fr* l_act,
                                  const Fr* y, int rot, uint32_t n) {
    const KnownFr ky = block_known(y);
    ZK_GRID_LOOP(i, n) {
        const uint32_t rn = rot_pow2(i, rot, n);
        Fr b = ld_elem<FrCfg>(betas);
        Fr l = fe_add_lazy<FrCfg>(ld_elem<FrCfg>(inputs[0] + i), b);
        Fr r = fe_add_lazy<FrCfg>(ld_elem<FrCfg>(tables[0] + i), b);
        for (int j = 1; j < group_len; j++) {
            b = ld_elem<FrCfg>(betas + j);
            l = fe_mul_lazy<FrCfg>(l, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(inputs[j] + i), b));
            r = fe_mul_lazy<FrCfg>(r, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(tables[j] + i), b));
        }
        Fr t = shuffle_tail(ld_elem<FrCfg>(res + i), ky, ld_elem<FrCfg>(z + i), ld_elem<FrCfg>(z + rn),
                            ld_elem<FrCfg>(l0 + i), ld_elem<FrCfg>(l_last + i), ld_elem<FrCfg>(l_act + i), l, r);
        st_elem<FrCfg>(res + i, t);
    }
}

cudaError_t shuffle_eval_h_v2(Fr* res, const Fr* const* inputs, const Fr* const* tables, const Fr* betas,
                              int group_len, const Fr* z, const Fr* l0, const Fr* l_last, const Fr* l_active_row,
                              const Fr* y, int rot, uint32_t n, cudaStream_t s) {
    if (n == 0 || group_len <= 0) return cudaSuccess;
    shuffle_v2_kernel<<<grid_for(n), 256, 0, s>>>(res, inputs, tables, betas, group_len, z, l0, l_last,
                                                  l_active_row, y, rot, n);
    return cudaGetLastError();
}

// --------------------------------------------------------------- small maps

// up to ZIP_KNOWN coefficients (the coset powers the quotient cycles through)
// are staged per block as known factors
static constexpr uint32_t ZIP_KNOWN = 64;

__global__ void mul_zip_kernel(Fr* buf, const Fr* coeff, uint32_t coeff_n, uint32_t n) {
    __shared__ KnownFr sk[ZIP_KNOWN];
    if (coeff_n <= ZIP_KNOWN) {
        for (uint32_t k = threadIdx.x; k < coeff_n; k += blockDim.x) sk[k] = known_fr(ld_elem<FrCfg>(coeff + k));
        __syncthreads();
        ZK_GRID_LOOP(i, n) st_elem<FrCfg>(buf + i, fe_canon<FrCfg>(mul_known(ld_elem<FrCfg>(buf + i), sk[i % coeff_n])));
        return;
    }
    ZK_GRID_LOOP(i, n) {
        st_elem<FrCfg>(buf + i, fe_mul<FrCfg>(ld_elem<FrCfg>(buf + i), ld_elem<FrCfg>(coeff + i % coeff_n)));
    }
}

cudaError_t field_mul_zip(Fr* buf, const Fr* coeff, uint32_t coeff_n, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (coeff_n == 0) return cudaErrorInvalidValue;
    mul_zip_kernel<<<grid_for(n), 256, 0, s>>>(buf, coeff, coeff_n, n);
    return cudaGetLastError();
}

// the constants c_j of up to SUM_KNOWN columns are staged per block as known
// factors; the sum stays lazily reduced until the store
static constexpr int SUM_KNOWN = 64;

__global__ void field_sum_kernel(Fr* res, Fr* const* v, Fr* const* v_c, const int* v_rot, const Fr* omegas,
                                 int v_n, uint32_t n) {
    __shared__ KnownFr sk[SUM_KNOWN];
    const bool staged = v_n <= SUM_KNOWN;
    if (staged) {
        for (int j = threadIdx.x; j < v_n; j += blockDim.x)
            if (v_c[j]) sk[j] = known_fr(ld_elem<FrCfg>(v_c[j]));
        __syncthreads();
    }
    ZK_GRID_LOOP(i, n) {
        Fr acc = fe_zero<FrCfg>();
        for (int j = 0; j < v_n; j++) {
            const uint32_t e = (uint32_t)(((long long)((int)n + v_rot[j]) * (long long)i) & (long long)(n - 1));
            Fr t = fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(v[j] + i), ld_elem<FrCfg>(omegas + e));
            if (v_c[j]) t = staged ? mul_known(t, sk[j]) : fe_mul_lazy<FrCfg>(t, ld_elem<FrCfg>(v_c[j]));
            acc = fe_add_lazy<FrCfg>(acc, t);
        }
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(acc));
    }
}

cudaError_t field_sum(Fr* res, Fr* const* v, Fr* const* v_c, const int* v_rot, const Fr* omegas, int v_n,
                      uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    field_sum_kernel<<<grid_for(n), 256, 0, s>>>(res, v, v_c, v_rot, omegas, v_n, n);
    return cudaGetLastError();
}

__global__ void shplonk_merge_kernel(Fr* res, const Fr* v, const Fr* values, const Fr* omegas, const Fr* diff,
                                     int nd, uint32_t n) {
    const KnownFr kv = block_known(v);
    ZK_GRID_LOOP(i, n) {
        Fr t = ld_elem<FrCfg>(values + i);
        const Fr w = ld_elem<FrCfg>(omegas + i);
        for (int j = 0; j < nd; j++) t = fe_mul_lazy<FrCfg>(t, fe_sub_lazy<FrCfg>(w, ld_elem<FrCfg>(diff + j)));
        st_elem<FrCfg>(res + i, fe_canon<FrCfg>(fe_add_lazy<FrCfg>(mul_known(ld_elem<FrCfg>(res + i), kv), t)));
    }
}

cudaError_t shplonk_h_x_merge(Fr* res, const Fr* v, const Fr* values, const Fr* omegas, const Fr* diff_points,
                              int diff_points_n, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    shplonk_merge_kernel<<<grid_for(n), 256, 0, s>>>(res, v, values, omegas, diff_points, diff_points_n, n);
    return cudaGetLastError();
}

}  // namespace zk
