// The quotient (h) phase of the prover over cosets of the extended domain, and
// the multi-open helpers the reference runs on the host.
//
// Reference behaviour replaced (src/eval_h.rs:410-586, 588-1199; its kernels
// cuda/bn254.cu:664-1071): every column involved in a constraint is extended
// to the whole 2^(k+e) domain (one NTT of 2^(k+e) per column, 1 GiB at
// k = 22), and each constraint family runs as its own kernel over those
// extended buffers, each re-reading and re-writing h; then h is multiplied by
// 1/Z_H, brought back by an iNTT of 2^(k+e) and the coset shift undone.
//
// Here the extended domain zeta <w_N> (N = E n, E = 2^e) is handled as its E
// cosets zeta w_N^j <w_n>, j < E: point m = j + E i of the extended domain is
// row i of coset j.  A rotation by r rows of the n-domain is a rotation by E r
// on the extended domain, i.e. by r rows inside the same coset, so every
// constraint of one coset reads that coset's rows only.  Per coset:
//   zkp_ntt_batch_twisted  the coset values of many coefficient columns at
//                          once: NTT_n of c_k (zeta w_N^j)^k;
//   zkp_eval_h_fused       every constraint (gates, permutation, logup
//                          lookups, shuffles) in one pass that reads each
//                          column once and writes h_j once, times 1/Z_H(coset j);
// and after the E cosets
//   zkp_coset_combine      from the E coset iNTTs of h to its 2^(k+e)
//                          coefficients: a radix-E inverse DFT across cosets
//                          per row, with the per-coset 1/Z_H, the w_N^-jr
//                          twist and the zeta^-m coset unshift folded in.
// The values equal the reference's to the bit: every step is exact field
// arithmetic, so any correct evaluation order gives the same canonical result.
//
// Multi-open helpers:
//   zkp_poly_divide_linear  q = (a(X) - a(z)) / (X - z), the division the
//                           reference runs on the host (src/multiopen.rs:
//                           145-159 GWC, 543-553 SHPLONK), as a scan:
//                           q_i = z^-i sum_{j>i} a_j z^(j-1);
//   zkp_poly_eval_batch     many polynomials at one point as dot products with
//                           the point's power table (src/eval_poly.rs:18-163
//                           evaluates one (polynomial, point) pair per call).
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "../../include/zkwasm_prover_kernel.h"

static inline const zk::Fr* CFr(const void* p) { return reinterpret_cast<const zk::Fr*>(p); }

namespace zk {

static __device__ __forceinline__ uint32_t rot_row(uint32_t i, int rot, uint32_t n) {
    return (uint32_t)((int64_t)i + rot) & (n - 1);
}

#define QZ_GRID_LOOP(i, n) \
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

static inline unsigned qz_grid(uint64_t n, unsigned tb) {
    uint64_t b = (n + tb - 1) / tb;
    if (b > 148u * 32u) b = 148u * 32u;
    return b ? (unsigned)b : 1u;
}

// ---------------------------------------------------------------- fused constraints

// Device-side view of zkp_eval_h_args (include/zkwasm_prover_kernel.h).
struct EvalHView {
    uint32_t n;
    int rot_scale;
    const Fr* y;
    const Fr* const* gate_terms;
    const int* gate_rots;
    int gate_terms_n;
    const Fr* l0;
    const Fr* l_last;
    const Fr* l_active;
    const Fr* x;
    const Fr* beta;
    const Fr* gamma;
    int perm_chunks;
    int perm_chunk_len;
    int perm_cols_n;
    int perm_last_rot;
    const Fr* const* perm_z;
    const Fr* const* perm_cols;
    const Fr* const* perm_sigmas;
    const Fr* perm_dbeta;
    int lookups;
    const Fr* const* lookup_cols;
    int shuffles;
    const Fr* const* shuffle_cols;
    const int* shuffle_group_len;
    const Fr* shuffle_betas;
    const Fr* scale;
};

// max permutation columns whose beta delta^c factors are staged per block
static constexpr int EVAL_H_MAX_PERM = 256;

__global__ void __launch_bounds__(256, 2) eval_h_fused_kernel(Fr* h, EvalHView a) {
    __shared__ KnownFr s_dbeta[EVAL_H_MAX_PERM];
    for (int c = threadIdx.x; c < a.perm_cols_n; c += blockDim.x) s_dbeta[c] = known_fr(ld_elem<FrCfg>(a.perm_dbeta + c));
    const KnownFr ky = block_known(a.y);
    const Fr one = fe_one<FrCfg>();
    const Fr beta = a.beta ? fe_canon<FrCfg>(ld_elem<FrCfg>(a.beta)) : fe_zero<FrCfg>();
    const Fr gamma = a.gamma ? fe_canon<FrCfg>(ld_elem<FrCfg>(a.gamma)) : fe_zero<FrCfg>();
    KnownFr kbeta = known_fr(beta);
    const uint32_t n = a.n;
    QZ_GRID_LOOP(i, n) {
        // gates: sum_t coeff_t prod_j col_tj[i + rot_tj]
        Fr acc = fe_zero<FrCfg>();
        {
            int vi = 0, ri = 0;
            while (vi < a.gate_terms_n) {
                Fr t = ld_elem<FrCfg>(a.gate_terms[vi++]);
                while (vi < a.gate_terms_n && a.gate_terms[vi]) {
                    t = fe_mul_lazy<FrCfg>(t, ld_elem<FrCfg>(a.gate_terms[vi] +
                                                             rot_row(i, a.gate_rots[ri] * a.rot_scale, n)));
                    vi++;
                    ri++;
                }
                acc = fe_add_lazy<FrCfg>(acc, t);
                vi++;
            }
        }
        const Fr l0 = ld_elem<FrCfg>(a.l0 + i);
        const Fr ll = ld_elem<FrCfg>(a.l_last + i);
        const Fr la = ld_elem<FrCfg>(a.l_active + i);
        if (a.perm_chunks > 0) {
            // l_0 (1 - z_0) and l_last (z_last^2 - z_last) (cuda/bn254.cu:664-699)
            const Fr z0 = ld_elem<FrCfg>(a.perm_z[0] + i);
            const Fr zl = ld_elem<FrCfg>(a.perm_z[a.perm_chunks - 1] + i);
            acc = mul_known(acc, ky);
            acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(l0, fe_sub_lazy<FrCfg>(one, z0)));
            acc = mul_known(acc, ky);
            acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(ll, fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(zl, zl), zl)));
            // chunk links l_0 (z_j - z_{j-1}(w^last X)) (cuda/bn254.cu:701-733)
            const uint32_t rp = rot_row(i, a.perm_last_rot * a.rot_scale, n);
            for (int j = 1; j < a.perm_chunks; j++) {
                acc = mul_known(acc, ky);
                const Fr d = fe_sub_lazy<FrCfg>(ld_elem<FrCfg>(a.perm_z[j] + i), ld_elem<FrCfg>(a.perm_z[j - 1] + rp));
                acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(d, l0));
            }
            // l_active (z(wX) prod (v + beta sigma + gamma) - z(X) prod (v + beta delta^c X + gamma))
            // (src/eval_h.rs:700-810)
            const Fr X = ld_elem<FrCfg>(a.x + i);
            const uint32_t rn = rot_row(i, a.rot_scale, n);
            int c = 0;
            for (int j = 0; j < a.perm_chunks; j++) {
                Fr L = ld_elem<FrCfg>(a.perm_z[j] + rn);
                Fr R = ld_elem<FrCfg>(a.perm_z[j] + i);
                const int end = c + a.perm_chunk_len < a.perm_cols_n ? c + a.perm_chunk_len : a.perm_cols_n;
                for (; c < end; c++) {
                    const Fr v = fe_add_lazy<FrCfg>(ld_elem<FrCfg>(a.perm_cols[c] + i), gamma);
                    const Fr bs = mul_known(ld_elem<FrCfg>(a.perm_sigmas[c] + i), kbeta);
                    L = fe_mul_lazy<FrCfg>(L, fe_add_lazy<FrCfg>(v, bs));
                    R = fe_mul_lazy<FrCfg>(R, fe_add_lazy<FrCfg>(v, mul_known(X, s_dbeta[c])));
                }
                acc = mul_known(acc, ky);
                acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(la, fe_sub_lazy<FrCfg>(L, R)));
            }
        }
        // logup lookups with one input per set (cuda/bn254.cu:867-921): with
        // f' = input + beta, t' = table + beta,
        // y^3 acc + y^2 l_0 z + y l_last z + l_active (((z(wX) - z) t' + m) f' - t')
        for (int k = 0; k < a.lookups; k++) {
            const Fr* const* q = a.lookup_cols + 4 * k;
            const Fr fb = fe_add_lazy<FrCfg>(ld_elem<FrCfg>(q[0] + i), beta);
            const Fr tb = fe_add_lazy<FrCfg>(ld_elem<FrCfg>(q[1] + i), beta);
            const Fr m = ld_elem<FrCfg>(q[2] + i);
            const Fr z = ld_elem<FrCfg>(q[3] + i);
            const Fr zn = ld_elem<FrCfg>(q[3] + rot_row(i, a.rot_scale, n));
            acc = mul_known(acc, ky);
            acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(l0, z));
            acc = mul_known(acc, ky);
            acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(ll, z));
            acc = mul_known(acc, ky);
            Fr u = fe_mul_lazy<FrCfg>(fe_sub_lazy<FrCfg>(zn, z), tb);
            u = fe_mul_lazy<FrCfg>(fe_add_lazy<FrCfg>(u, m), fb);
            u = fe_sub_lazy<FrCfg>(u, tb);
            acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(u, la));
        }
        // shuffles (cuda/bn254.cu:1017-1071): with l = prod (input_g + beta_g),
        // r = prod (table_g + beta_g),
        // y^3 acc + y^2 l_0 (1 - z) + y l_last (z^2 - z) + l_active (r z(wX) - l z)
        {
            int off = 0;
            for (int s = 0; s < a.shuffles; s++) {
                const Fr* const* q = a.shuffle_cols + off;
                const int g = a.shuffle_group_len[s];
                const Fr z = ld_elem<FrCfg>(q[0] + i);
                const Fr zn = ld_elem<FrCfg>(q[0] + rot_row(i, a.rot_scale, n));
                Fr l = one, r = one;
                for (int t = 0; t < g; t++) {
                    const Fr bt = ld_elem<FrCfg>(a.shuffle_betas + t);
                    l = fe_mul_lazy<FrCfg>(l, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(q[1 + 2 * t] + i), bt));
                    r = fe_mul_lazy<FrCfg>(r, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(q[2 + 2 * t] + i), bt));
                }
                acc = mul_known(acc, ky);
                acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(l0, fe_sub_lazy<FrCfg>(one, z)));
                acc = mul_known(acc, ky);
                acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(ll, fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(z, z), z)));
                acc = mul_known(acc, ky);
                const Fr u = fe_sub_lazy<FrCfg>(fe_mul_lazy<FrCfg>(r, zn), fe_mul_lazy<FrCfg>(l, z));
                acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(u, la));
                off += 1 + 2 * g;
            }
        }
        if (a.scale) acc = fe_mul_lazy<FrCfg>(acc, ld_elem<FrCfg>(a.scale));
        st_elem<FrCfg>(h + i, fe_canon<FrCfg>(acc));
    }
}

// ---------------------------------------------------------------- coset combine

// out[r + n s] = zeta^-(r + n s) / E * sum_j w_E^-(j s) t_j w_N^-(j r) g_j[r]
// (g_j: the inverse n-point transform of coset j's values, scaled by 1/n).
// consts: t_0..t_{E-1}, then w_E^-k for k < E, then zeta^-k / E for k < 3.
template <int E>
__global__ void __launch_bounds__(256) coset_combine_kernel(Fr* out, const Fr* g, size_t g_stride, const Fr* winv,
                                                            const Fr* consts, uint32_t n) {
    __shared__ Fr c[E + E + 3];
    for (int k = threadIdx.x; k < 2 * E + 3; k += blockDim.x) c[k] = ld_elem<FrCfg>(consts + k);
    __syncthreads();
    QZ_GRID_LOOP(r, n) {
        Fr x[E];
        const Fr w = ld_elem<FrCfg>(winv + r);
        Fr p = fe_one<FrCfg>();
        for (int j = 0; j < E; j++) {
            Fr v = fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(g + (size_t)j * g_stride + r), c[j]);
            if (j) v = fe_mul_lazy<FrCfg>(v, p);
            x[j] = v;
            if (j + 1 < E) p = j ? fe_mul_lazy<FrCfg>(p, w) : w;
        }
        const uint32_t m3 = r % 3u, n3 = n % 3u;
        for (int s = 0; s < E; s++) {
            Fr acc = x[0];
            for (int j = 1; j < E; j++) acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(x[j], c[E + ((j * s) % E)]));
            const uint32_t k = (m3 + n3 * (uint32_t)s) % 3u;
            st_elem<FrCfg>(out + r + (size_t)n * s, fe_mul<FrCfg>(fe_canon<FrCfg>(acc), c[2 * E + k]));
        }
    }
}

// ---------------------------------------------------------------- linear division and evaluation

// b_j = a_j p_j for j >= 1 (p_j = z^(j-1)), b_0 = 0
__global__ void ruffini_weight_kernel(Fr* b, const Fr* a, const Fr* p, uint32_t n) {
    QZ_GRID_LOOP(j, n) {
        st_elem<FrCfg>(b + j, j ? fe_mul<FrCfg>(ld_elem<FrCfg>(a + j), ld_elem<FrCfg>(p + j - 1)) : fe_zero<FrCfg>());
    }
}

// q_i = (total - prefix_i - b_i) zinv^i for i < n - 1, q_{n-1} = 0; prefix is
// the exclusive prefix sum of b, total = prefix_{n-1} + b_{n-1}
__global__ void ruffini_finish_kernel(Fr* q, const Fr* prefix, const Fr* b, const Fr* zinv_pow, uint32_t n) {
    const Fr total = fe_add<FrCfg>(ld_elem<FrCfg>(prefix + n - 1), ld_elem<FrCfg>(b + n - 1));
    QZ_GRID_LOOP(i, n) {
        if (i == n - 1) {
            st_elem<FrCfg>(q + i, fe_zero<FrCfg>());
        } else {
            const Fr s = fe_sub<FrCfg>(fe_sub<FrCfg>(total, ld_elem<FrCfg>(prefix + i)), ld_elem<FrCfg>(b + i));
            st_elem<FrCfg>(q + i, fe_mul<FrCfg>(s, ld_elem<FrCfg>(zinv_pow + i)));
        }
    }
}

__global__ void shift_down_kernel(Fr* q, const Fr* a, uint32_t n) {
    QZ_GRID_LOOP(i, n) { st_elem<FrCfg>(q + i, i + 1 < n ? ld_elem<FrCfg>(a + i + 1) : fe_zero<FrCfg>()); }
}

// partial dot products: block b of polynomial p sums poly[i] pw[i] over its
// stride of rows into part[p * nb + b]
__global__ void __launch_bounds__(256) dot_partial_kernel(Fr* part, const Fr* const* polys, const Fr* pw, uint32_t n,
                                                          uint32_t nb) {
    __shared__ Fr red[256];
    const Fr* poly = polys[blockIdx.y];
    Fr acc = fe_zero<FrCfg>();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nb * blockDim.x)
        acc = fe_add_lazy<FrCfg>(acc, fe_mul_lazy<FrCfg>(ld_elem<FrCfg>(poly + i), ld_elem<FrCfg>(pw + i)));
    red[threadIdx.x] = fe_canon<FrCfg>(acc);
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] = fe_add<FrCfg>(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) st_elem<FrCfg>(part + (size_t)blockIdx.y * nb + blockIdx.x, red[0]);
}

__global__ void dot_final_kernel(Fr* out, const Fr* part, uint32_t nb, uint32_t count) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    Fr acc = fe_zero<FrCfg>();
    for (uint32_t b = 0; b < nb; b++) acc = fe_add<FrCfg>(acc, ld_elem<FrCfg>(part + (size_t)p * nb + b));
    st_elem<FrCfg>(out + p, acc);
}

}  // namespace zk

using namespace zk;

static constexpr uint32_t DOT_BLOCKS = 64;

extern "C" {

cudaError_t zkp_ntt_batch_twisted(void* out, const void* in, void* tmp, const void* omegas, const void* in_mul,
                                  const void* scale, int log_n, uint32_t ncols, size_t in_stride, size_t out_stride,
                                  int pairs, cudaStream_t stream) {
    if (log_n < 1 || log_n > 28 || !out || !in || !omegas || ncols == 0 || ncols > 65535) return cudaErrorInvalidValue;
    const size_t n = (size_t)1 << log_n;
    if (in_stride < n || out_stride < n || out == in) return cudaErrorInvalidValue;
    int rad[4];
    const int np = ntt_plan(log_n, rad);
    if (np > 1 && !tmp) return cudaErrorInvalidValue;
    // the last pass writes `out`; earlier passes alternate out / tmp back from it
    const Fr* src = reinterpret_cast<const Fr*>(in);
    size_t src_stride = in_stride;
    int log_p = 0;
    for (int p = 0; p < np; p++) {
        const bool to_out = ((np - 1 - p) % 2) == 0;
        Fr* dst = to_out ? reinterpret_cast<Fr*>(out) : reinterpret_cast<Fr*>(tmp);
        NttPassArgs a = {};
        a.src = src;
        a.dst = dst;
        a.tw = reinterpret_cast<const Fr*>(omegas);
        a.log_n = log_n;
        a.log_p = log_p;
        a.in_mul = p == 0 ? reinterpret_cast<const Fr*>(in_mul) : nullptr;
        a.scale = p == np - 1 ? reinterpret_cast<const Fr*>(scale) : nullptr;
        a.src_ys = src_stride;
        a.dst_ys = to_out ? out_stride : n;
        a.pairs = pairs ? 1 : 0;
        ZK_CHECK(ntt_pass(a, rad[p], ncols, 1, stream));
        src = dst;
        src_stride = a.dst_ys;
        log_p += rad[p];
    }
    return cudaGetLastError();
}

cudaError_t zkp_eval_h_fused(void* h, const zkp_eval_h_args* args, cudaStream_t stream) {
    if (!h || !args) return cudaErrorInvalidValue;
    const zkp_eval_h_args& g = *args;
    const uint32_t n = g.n;
    if (n == 0) return cudaSuccess;
    if ((n & (n - 1)) != 0 || !g.y || !g.l0 || !g.l_last || !g.l_active) return cudaErrorInvalidValue;
    if (g.gate_terms_n < 0 || (g.gate_terms_n > 0 && (!g.gate_terms || !g.gate_rots))) return cudaErrorInvalidValue;
    if (g.perm_chunks < 0 || g.lookups < 0 || g.shuffles < 0) return cudaErrorInvalidValue;
    if (g.perm_chunks > 0 &&
        (!g.perm_z || !g.perm_cols || !g.perm_sigmas || !g.perm_dbeta || !g.x || !g.beta || !g.gamma ||
         g.perm_chunk_len <= 0 || g.perm_cols_n <= 0 || g.perm_cols_n > EVAL_H_MAX_PERM ||
         (g.perm_cols_n + g.perm_chunk_len - 1) / g.perm_chunk_len != g.perm_chunks))
        return cudaErrorInvalidValue;
    if (g.lookups > 0 && (!g.lookup_cols || !g.beta)) return cudaErrorInvalidValue;
    if (g.shuffles > 0 && (!g.shuffle_cols || !g.shuffle_group_len || !g.shuffle_betas)) return cudaErrorInvalidValue;
    EvalHView v;
    v.n = n;
    v.rot_scale = g.rot_scale ? g.rot_scale : 1;
    v.y = CFr(g.y);
    v.gate_terms = reinterpret_cast<const Fr* const*>(g.gate_terms);
    v.gate_rots = reinterpret_cast<const int*>(g.gate_rots);
    v.gate_terms_n = g.gate_terms_n;
    v.l0 = CFr(g.l0);
    v.l_last = CFr(g.l_last);
    v.l_active = CFr(g.l_active);
    v.x = CFr(g.x);
    v.beta = CFr(g.beta);
    v.gamma = CFr(g.gamma);
    v.perm_chunks = g.perm_chunks;
    v.perm_chunk_len = g.perm_chunk_len;
    v.perm_cols_n = g.perm_chunks > 0 ? g.perm_cols_n : 0;
    v.perm_last_rot = g.perm_last_rot;
    v.perm_z = reinterpret_cast<const Fr* const*>(g.perm_z);
    v.perm_cols = reinterpret_cast<const Fr* const*>(g.perm_cols);
    v.perm_sigmas = reinterpret_cast<const Fr* const*>(g.perm_sigmas);
    v.perm_dbeta = CFr(g.perm_dbeta);
    v.lookups = g.lookups;
    v.lookup_cols = reinterpret_cast<const Fr* const*>(g.lookup_cols);
    v.shuffles = g.shuffles;
    v.shuffle_cols = reinterpret_cast<const Fr* const*>(g.shuffle_cols);
    v.shuffle_group_len = reinterpret_cast<const int*>(g.shuffle_group_len);
    v.shuffle_betas = CFr(g.shuffle_betas);
    v.scale = CFr(g.scale);
    eval_h_fused_kernel<<<qz_grid(n, 256), 256, 0, stream>>>(reinterpret_cast<Fr*>(h), v);
    return cudaGetLastError();
}

cudaError_t zkp_coset_combine(void* out, const void* g, size_t g_stride, const void* winv, const void* consts,
                              int log_n, int ext_bits, cudaStream_t stream) {
    if (!out || !g || !winv || !consts || log_n < 1 || log_n > 28) return cudaErrorInvalidValue;
    const uint32_t n = 1u << log_n;
    if (g_stride < n) return cudaErrorInvalidValue;
    Fr* o = reinterpret_cast<Fr*>(out);
    const Fr* gg = CFr(g);
    const Fr* w = CFr(winv);
    const Fr* c = CFr(consts);
    const unsigned grid = qz_grid(n, 256);
    switch (ext_bits) {
        case 1: coset_combine_kernel<2><<<grid, 256, 0, stream>>>(o, gg, g_stride, w, c, n); break;
        case 2: coset_combine_kernel<4><<<grid, 256, 0, stream>>>(o, gg, g_stride, w, c, n); break;
        case 3: coset_combine_kernel<8><<<grid, 256, 0, stream>>>(o, gg, g_stride, w, c, n); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t zkp_shoup_pairs(void* out, const void* in, uint32_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (!out || !in || out == in) return cudaErrorInvalidValue;
    return shoup_pairs(reinterpret_cast<Fr*>(out), CFr(in), n, stream);
}

size_t zkp_poly_divide_scratch_elems(uint32_t n) { return 4 * (size_t)n + fr_scan_tmp_elems(n); }

cudaError_t zkp_poly_divide_linear(void* q, const void* a, const void* z, uint32_t n, void* scratch,
                                   cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (!q || !a || !z || !scratch || q == a) return cudaErrorInvalidValue;
    Fr zm = *reinterpret_cast<const Fr*>(z);
    zm = fe_canon<FrCfg>(zm);
    bool zero = true;
    for (int k = 0; k < 8; k++) zero = zero && zm.v[k] == 0;
    if (zero) {
        shift_down_kernel<<<qz_grid(n, 256), 256, 0, stream>>>(reinterpret_cast<Fr*>(q), CFr(a), n);
        return cudaGetLastError();
    }
    const Fr zinv = fe_inv<FrCfg>(zm);
    Fr* s = reinterpret_cast<Fr*>(scratch);
    Fr* pz = s;             // z^j, j < n, then zinv^i
    Fr* b = s + n;          // weighted coefficients
    Fr* pre = s + 2 * (size_t)n;  // exclusive prefix sums of b
    Fr* consts = s + 3 * (size_t)n;  // z, zinv
    Fr* tmp = s + 4 * (size_t)n;
    Fr hc[2] = {zm, zinv};
    ZK_CHECK(cudaMemcpyAsync(consts, hc, sizeof(hc), cudaMemcpyHostToDevice, stream));
    ZK_CHECK(geometric(pz, nullptr, consts, n, stream));
    ruffini_weight_kernel<<<qz_grid(n, 256), 256, 0, stream>>>(b, CFr(a), pz, n);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(fr_scan_excl(pre, b, n, nullptr, 0, tmp, stream));
    ZK_CHECK(geometric(pz, nullptr, consts + 1, n, stream));
    ruffini_finish_kernel<<<qz_grid(n, 256), 256, 0, stream>>>(reinterpret_cast<Fr*>(q), pre, b, pz, n);
    return cudaGetLastError();
}

size_t zkp_poly_eval_batch_scratch_elems(uint32_t count) { return (size_t)count * DOT_BLOCKS; }

cudaError_t zkp_poly_eval_batch(void* out, const void* polys, uint32_t count, const void* powers, uint32_t n,
                                void* scratch, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    if (!out || !polys || !powers || !scratch || n == 0 || count > 65535) return cudaErrorInvalidValue;
    dim3 grid(DOT_BLOCKS, count);
    dot_partial_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<Fr*>(scratch),
                                                 reinterpret_cast<const Fr* const*>(polys), CFr(powers), n,
                                                 DOT_BLOCKS);
    ZK_CHECK(cudaGetLastError());
    dot_final_kernel<<<(count + 127) / 128, 128, 0, stream>>>(reinterpret_cast<Fr*>(out),
                                                              reinterpret_cast<const Fr*>(scratch), DOT_BLOCKS, count);
    return cudaGetLastError();
}

}  // extern "C"
