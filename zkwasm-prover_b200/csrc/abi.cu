// extern "C" entry points: the reference-compatible symbols of
// include/zkwasm_prover_kernel.h (src/cuda/bn254_c.rs:4-309) and the batched
// zkp_* API.  Thin argument adapters over the kernels in this directory.
#include "common.cuh"
#include "kernels.h"
#include "../../include/zkwasm_prover_kernel.h"

using namespace zk;

#include <initializer_list>

static inline Fr* F(void* p) { return reinterpret_cast<Fr*>(p); }

// Argument checks of the reference-compatible symbols: every pointer a kernel
// dereferences must be set once there is work (n > 0).  A failed check
// returns cudaErrorInvalidValue before anything is enqueued.
static inline bool all_set(std::initializer_list<const void*> ps) {
    for (const void* q : ps)
        if (!q) return false;
    return true;
}
static inline const Fr* CF(const void* p) { return reinterpret_cast<const Fr*>(p); }

// ------------------------------------------------------------------ kernels used only here

namespace zk {

// twist[j * n + k] = (shift * w_ext^j)^k (as Montgomery elements or pairs)
template <bool PAIRS>
__global__ void twist_kernel(Fr* twist, const Fr* shift, const Fr* w_ext, uint32_t n, uint32_t chunk) {
    const uint32_t j = blockIdx.y;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = t * chunk, e = s + chunk;
    if (e > n) e = n;
    if (s >= e) return;
    const Fr base = fe_mul<FrCfg>(ld_elem<FrCfg>(shift), fe_pow_u32<FrCfg>(ld_elem<FrCfg>(w_ext), j));
    Fr cur = fe_pow_u32<FrCfg>(base, s);
    for (uint32_t i = s; i < e; i++) {
        st_factor<PAIRS>(twist, (size_t)j * n + i, cur);
        cur = fe_mul<FrCfg>(cur, base);
    }
}

__global__ void to_mont_kernel(Fr* out, const Fr* in, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) st_elem<FrCfg>(out + i, fe_to_mont<FrCfg>(ld_elem<FrCfg>(in + i)));
}

// out[i] = [k_i] G (affine, Montgomery form) for 64-bit k_i; G = (1, 2)
__global__ void g1_multiples_kernel(Aff* out, const uint64_t* k64, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = k64[i];
    Fq g1 = fe_zero<FqCfg>(), g2 = fe_zero<FqCfg>();
    g1.v[0] = 1;
    g2.v[0] = 2;
    g1 = fe_to_mont<FqCfg>(g1);
    g2 = fe_to_mont<FqCfg>(g2);
    Xyzz acc = xyzz_identity();
    for (int b = 63; b >= 0; b--) {
        acc = xyzz_dbl(acc);
        if ((k >> b) & 1) acc = xyzz_add_aff(acc, g1, g2);
    }
    Aff a;
    if (xyzz_is_id(acc)) {
        a.x = fe_zero<FqCfg>();
        a.y = fe_zero<FqCfg>();
    } else {
        const Fq inv = fe_inv<FqCfg>(fe_mul<FqCfg>(acc.zz, acc.zzz));
        a.x = fe_mul<FqCfg>(fe_mul<FqCfg>(acc.x, acc.zzz), inv);
        a.y = fe_mul<FqCfg>(fe_mul<FqCfg>(acc.y, acc.zz), inv);
    }
    st_elem<FqCfg>(&out[i].x, a.x);
    st_elem<FqCfg>(&out[i].y, a.y);
}

}  // namespace zk

extern "C" {

// ================================================================== Part 1

cudaError_t ntt(void* buf, void* tmp, void* pq, void* omega, void* n_inv, int array_log, int max_deg, void* swap,
                cudaStream_t stream) {
    (void)pq;
    (void)max_deg;
    if (array_log < 0 || array_log > 28 || !buf || !omega || !swap) return cudaErrorInvalidValue;
    bool in_tmp = false;
    if (array_log > 0) {
        if (!tmp && array_log > 12) return cudaErrorInvalidValue;
        ZK_CHECK(ntt_run(F(buf), F(tmp), CF(omega), CF(n_inv), array_log, 1, 0, &in_tmp, stream));
    } else if (n_inv) {
        // n = 1: the transform is the identity, n^-1 = 1
    }
    *reinterpret_cast<bool*>(swap) = in_tmp;
    return cudaGetLastError();
}

cudaError_t field_op(void* res, void* l, int l_rot, void* l_c, void* r, int r_rot, void* r_c, int size, int op,
                     cudaStream_t stream) {
    if (size < 0 || op < 0 || op > 3) return cudaErrorInvalidValue;
    // L is l (times l_c) or l_c alone; R likewise, and unused by op 2
    if (size > 0 && (!res || (!l && !l_c) || (op != 2 && !r && !r_c))) return cudaErrorInvalidValue;
    return zk::field_op(F(res), CF(l), l_rot, CF(l_c), CF(r), r_rot, CF(r_c), (uint32_t)size, op, stream);
}

cudaError_t extended_prepare(void* s, void* coset_powers, int coset_powers_n, int size, int extended_size,
                             int to_coset, cudaStream_t stream) {
    if (size < 0 || extended_size < 0 || coset_powers_n <= 0) return cudaErrorInvalidValue;
    if (!to_coset && size > extended_size) return cudaErrorInvalidValue;
    if ((to_coset ? extended_size : (extended_size > size ? extended_size : size)) > 0 &&
        (!s || (coset_powers_n > 1 && !coset_powers)))
        return cudaErrorInvalidValue;
    return zk::extended_prepare(F(s), CF(coset_powers), (uint32_t)coset_powers_n, (uint32_t)size,
                                (uint32_t)extended_size, to_coset, stream);
}

cudaError_t permutation_eval_h_p1(void* res, void* first_set, void* last_set, void* l0, void* l_last, void* y,
                                  int n) {
    if (n < 0 || (n > 0 && !all_set({res, first_set, last_set, l0, l_last, y}))) return cudaErrorInvalidValue;
    return zk::permutation_eval_h_p1(F(res), CF(first_set), CF(last_set), CF(l0), CF(l_last), CF(y), (uint32_t)n, 0);
}

cudaError_t permutation_eval_h_p2(void* res, void* set, void* l0, void* l_last, void* y, int n_set, int rot, int n) {
    (void)l_last;
    if (n < 0 || n_set < 0 || (n > 0 && n_set > 1 && !all_set({res, set, l0, y}))) return cudaErrorInvalidValue;
    return zk::permutation_eval_h_p2(F(res), reinterpret_cast<const Fr* const*>(set), CF(l0), CF(y), n_set, rot,
                                     (uint32_t)n, 0);
}

cudaError_t permutation_eval_h_l(void* res, void* beta, void* gamma, void* p, int n, cudaStream_t stream) {
    if (n < 0 || (n > 0 && !all_set({res, beta, gamma, p}))) return cudaErrorInvalidValue;
    return zk::permutation_eval_h_l(F(res), CF(beta), CF(gamma), CF(p), (uint32_t)n, stream);
}

cudaError_t field_sum(void* res, void* v, void* v_c, void* v_rot, void* omegas, int v_n, int n) {
    if (n < 0 || v_n < 0 || (n > 0 && (!res || (v_n > 0 && !all_set({v, v_c, v_rot, omegas})))))
        return cudaErrorInvalidValue;
    return zk::field_sum(F(res), reinterpret_cast<Fr* const*>(v), reinterpret_cast<Fr* const*>(v_c),
                         reinterpret_cast<const int*>(v_rot), CF(omegas), v_n, (uint32_t)n, 0);
}

cudaError_t field_op_batch_mul_sum(void* res, void* v, void* rot, int v_n, int n, cudaStream_t stream) {
    if (n < 0 || v_n < 0 || (n > 0 && v_n > 0 && !all_set({res, v, rot}))) return cudaErrorInvalidValue;
    return zk::field_op_batch_mul_sum(F(res), reinterpret_cast<Fr* const*>(v), reinterpret_cast<const int*>(rot),
                                      v_n, (uint32_t)n, stream);
}

cudaError_t lookup_eval_h(void* res, void* input, void* table, void* permuted_input, void* permuted_table, void* z,
                          void* l0, void* l_last, void* l_active_row, void* y, void* beta, void* gamma, int rot,
                          int n, cudaStream_t stream) {
    if (n < 0 || (n > 0 && !all_set({res, input, table, permuted_input, permuted_table, z, l0, l_last, l_active_row, y,
                                      beta, gamma})))
        return cudaErrorInvalidValue;
    return zk::lookup_eval_h(F(res), CF(input), CF(table), CF(permuted_input), CF(permuted_table), CF(z), CF(l0),
                             CF(l_last), CF(l_active_row), CF(y), CF(beta), CF(gamma), rot, (uint32_t)n, stream);
}

cudaError_t logup_eval_h(void* res, void* input_product, void* input_product_sum, void* table, void* multiplicity,
                         void* z_first, void* z_last, void* l0, void* l_last, void* l_active_row, void* y, int rot,
                         int n, cudaStream_t stream) {
    if (n < 0 || (n > 0 && !all_set({res, input_product, input_product_sum, table, multiplicity, z_first, z_last, l0,
                                      l_last, l_active_row, y})))
        return cudaErrorInvalidValue;
    return zk::logup_eval_h(F(res), CF(input_product), CF(input_product_sum), CF(table), CF(multiplicity),
                            CF(z_first), CF(z_last), CF(l0), CF(l_last), CF(l_active_row), CF(y), rot, (uint32_t)n,
                            stream);
}

cudaError_t logup_eval_h_extra_inputs(void* res, void* input_product, void* input_product_sum, void* z,
                                      void* l_active_row, void* y, int rot, int n, cudaStream_t stream) {
    if (n < 0 || (n > 0 && !all_set({res, input_product, input_product_sum, z, l_active_row, y})))
        return cudaErrorInvalidValue;
    return zk::logup_eval_h_extra_inputs(F(res), CF(input_product), CF(input_product_sum), CF(z), CF(l_active_row),
                                         CF(y), rot, (uint32_t)n, stream);
}

cudaError_t logup_eval_h_z_set(void* res, void* set, void* l0, void* l_last, void* y, int n_set, int rot, int n,
                               cudaStream_t stream) {
    (void)l_last;
    if (n < 0 || n_set < 0 || (n > 0 && n_set > 1 && !all_set({res, set, l0, y}))) return cudaErrorInvalidValue;
    return zk::permutation_eval_h_p2(F(res), reinterpret_cast<const Fr* const*>(set), CF(l0), CF(y), n_set, rot,
                                     (uint32_t)n, stream);
}

cudaError_t logup_sum_input_inv(void* sum, void* input, void* temp, void* beta, int init, int n,
                                cudaStream_t stream) {
    if (n < 0 || (n > 0 && !all_set({sum, input, beta}))) return cudaErrorInvalidValue;
    // temp: the host's n-element buffer (src/lib.rs:596), scratch of the
    // three-phase inversion
    return zk::batch_inverse(F(sum), CF(input), CF(beta), (uint32_t)n, init != 0, F(temp), temp ? (size_t)n : 0,
                             stream);
}

cudaError_t logup_eval_h_inputs_product_sum(void* product, void* product_sum, void* sets, int n_set, int n,
                                            cudaStream_t stream) {
    if (n < 0 || n_set < 1 || (n > 0 && !all_set({product, product_sum, sets}))) return cudaErrorInvalidValue;
    return zk::logup_eval_h_inputs_product_sum(F(product), F(product_sum), reinterpret_cast<const Fr* const*>(sets),
                                               n_set, (uint32_t)n, stream);
}

cudaError_t shuffle_eval_h(void* res, void* input, void* table, void* z, void* l0, void* l_last, void* l_active_row,
                           void* y, int rot, int n) {
    if (n < 0 || (n > 0 && !all_set({res, input, table, z, l0, l_last, l_active_row, y}))) return cudaErrorInvalidValue;
    return zk::shuffle_eval_h(F(res), CF(input), CF(table), CF(z), CF(l0), CF(l_last), CF(l_active_row), CF(y), rot,
                              (uint32_t)n, 0);
}

cudaError_t shuffle_eval_h_v2(void* res, void* inputs, void* tables, void* betas, int group_len, void* z, void* l0,
                              void* l_last, void* l_active_row, void* y, int rot, int n) {
    if (n < 0 || group_len < 1 ||
        (n > 0 && !all_set({res, inputs, tables, betas, z, l0, l_last, l_active_row, y})))
        return cudaErrorInvalidValue;
    return zk::shuffle_eval_h_v2(F(res), reinterpret_cast<const Fr* const*>(inputs),
                                 reinterpret_cast<const Fr* const*>(tables), CF(betas), group_len, CF(z), CF(l0),
                                 CF(l_last), CF(l_active_row), CF(y), rot, (uint32_t)n, 0);
}

cudaError_t expand_omega_buffer(void* buf, int n, int may_bit_reversed) {
    (void)may_bit_reversed;
    if (n < 0 || n > 30 || !buf) return cudaErrorInvalidValue;
    return zk::expand_powers(F(buf), 1u << n, 0);
}

cudaError_t field_mul_zip(void* buf, void* coeff, int coeff_n, int n) {
    if (n < 0 || coeff_n <= 0 || (n > 0 && !all_set({buf, coeff}))) return cudaErrorInvalidValue;
    return zk::field_mul_zip(F(buf), CF(coeff), (uint32_t)coeff_n, (uint32_t)n, 0);
}

cudaError_t poly_eval(void* p, void* res, void* x, int n, cudaStream_t stream) {
    if (n <= 0 || (n & (n - 1)) != 0 || !all_set({p, res, x})) return cudaErrorInvalidValue;
    return zk::poly_eval(CF(p), F(res), CF(x), (uint32_t)n, stream);
}

cudaError_t shplonk_h_x_merge(void* res, void* v, void* values, void* omegas, void* diff_points, int diff_points_n,
                              int n) {
    if (n < 0 || diff_points_n < 0 ||
        (n > 0 && (!all_set({res, v, values, omegas}) || (diff_points_n > 0 && !diff_points))))
        return cudaErrorInvalidValue;
    return zk::shplonk_h_x_merge(F(res), CF(v), CF(values), CF(omegas), CF(diff_points), diff_points_n, (uint32_t)n,
                                 0);
}

cudaError_t shplonk_h_x_div_points(void* values, void* omegas, void* points, int points_n, int n) {
    if (n < 0 || points_n < 0 || (n > 0 && (!all_set({values, omegas}) || (points_n > 0 && !points))))
        return cudaErrorInvalidValue;
    return zk::div_by_point_diffs(F(values), CF(omegas), CF(points), points_n, (uint32_t)n, nullptr, 0, 0);
}

cudaError_t eval_logup_z_compose(void* z, void* input, void* table, void* multiplicity, void* beta, void* last_z,
                                 int last_z_index, int n, cudaStream_t stream) {
    if (n <= 0 || last_z_index < 0 || last_z_index >= n || !all_set({z, input, table, multiplicity, beta, last_z}))
        return cudaErrorInvalidValue;
    return zk::logup_z_compose(F(z), CF(input), CF(table), CF(multiplicity), CF(beta), F(last_z), last_z_index,
                               (uint32_t)n, F(table), stream);
}

cudaError_t eval_logup_z_pure(void* z, void* input, void* table, void* last_z, int last_z_index, int n,
                              cudaStream_t stream) {
    (void)input;
    if (n <= 0 || last_z_index < 0 || last_z_index >= n || !all_set({z, table, last_z})) return cudaErrorInvalidValue;
    return zk::logup_z_scan(F(z), F(last_z), last_z_index, (uint32_t)n, F(table), stream);
}

// byte offset, inside the 256-byte head of each MSM region, of the note msm()
// leaves for batch_msm_collect (the Jacobian result takes bytes 0..95)
static constexpr uint32_t MSM_NOTE_OFF = 128;

cudaError_t batch_msm_collect(void* remain_indices, void* remain_acc, void* next_remain_indices,
                              void* next_remain_acc, void* buckets, uint32_t workers, uint32_t windows,
                              uint32_t window_bits, uint32_t batch_size, cudaStream_t stream) {
    (void)remain_indices;
    (void)remain_acc;
    (void)next_remain_indices;
    (void)next_remain_acc;
    (void)workers;
    (void)windows;
    (void)window_bits;
    if (batch_size > 0 && !buckets) return cudaErrorInvalidValue;
    ZK_CHECK(cudaGetLastError());  // errors of earlier msm() launches surface here, as in the reference
    if (batch_size == 0) return cudaSuccess;
    // buckets: device array of the per-MSM regions msm() parked its window sums in
    return msm_collect(reinterpret_cast<char* const*>(buckets), batch_size, MSM_NOTE_OFF, stream);
}

cudaError_t msm(void* res, void* p, void* s, void* indices_buf0, void* indices_buf1, void* indices_buf2,
                void* indices_buf3, void* sort_buf, void* indices_buf, int array_len, int windows, int window_bits,
                int threads, int workers, int prepared_sort_indices_temp_storage_bytes, int skip_zero,
                cudaStream_t stream) {
    (void)indices_buf0;
    (void)indices_buf1;
    (void)indices_buf2;
    (void)indices_buf3;
    (void)indices_buf;
    (void)threads;
    (void)prepared_sort_indices_temp_storage_bytes;
    (void)skip_zero;
    if (array_len < 0 || windows <= 0 || window_bits <= 0 || window_bits > 24 || workers < 0 || !res || !sort_buf)
        return cudaErrorInvalidValue;
    if (array_len > 0 && (!p || !s)) return cudaErrorInvalidValue;
    const uint32_t n = (uint32_t)array_len;
    // scratch the reference host allocates for this call (src/cuda/msm.rs:297-317)
    const size_t words_avail = (size_t)3 * n * (size_t)windows;
    const size_t region_bytes = (((size_t)windows << window_bits) + 2 * (size_t)workers) * sizeof(Jac);
    const size_t head = 256;  // res[0] (the result) and the parked note stay clear of the scratch points
    if (region_bytes <= head) return cudaErrorInvalidValue;
    // Whole 254-bit scalars, no GLV split: with the final combinations of all
    // columns running side by side in batch_msm_collect, halving the final's
    // doublings gains nothing and the split and the endomorphism images cost.
    // Preferred window first, then wider and narrower ones until the plan fits.
    const int c0 = msm_make_plan(n, 0, false).c;
    int order[40];
    int no = 0;
    order[no++] = c0;
    for (int d = 1; d < 20; d++) {
        if (c0 + d <= 22) order[no++] = c0 + d;
        if (c0 - d >= 4) order[no++] = c0 - d;
    }
    // both caller buffers are scratch arenas: the sort buffer (shared by every
    // msm() call of a batch) and the region after its 256-byte head, which
    // must hold the window sums that batch_msm_collect reads later
    void* arena[2] = {sort_buf, reinterpret_cast<char*>(res) + head};
    const size_t arena_bytes[2] = {words_avail * 4, region_bytes - head};
    for (int i = 0; i < no; i++) {
        MsmPlan pl = msm_make_plan(n, order[i], false);
        MsmScratch sc = {};
        if (msm_layout_arenas(pl, arena, arena_bytes, 2, &sc, 1))
            // the final combination runs in batch_msm_collect, for all MSMs at once
            return msm_run(reinterpret_cast<Jac*>(res), reinterpret_cast<const Aff*>(p), CF(s), pl, sc, stream,
                           reinterpret_cast<char*>(res) + MSM_NOTE_OFF);
    }
    return cudaErrorInvalidValue;
}

cudaError_t prepare_table_lookup(void* table, void* table_lowest_u32, void* sorted_table_lowest_u32, void* index,
                                 void* sorted_index, void* start_offset, void* candidate_sort_temp_storage,
                                 uint32_t candidate_sort_temp_storage_bytes, uint32_t k, uint32_t unusable_rows_start,
                                 cudaStream_t stream) {
    (void)table_lowest_u32;
    (void)sorted_table_lowest_u32;
    (void)index;
    (void)sorted_index;
    (void)candidate_sort_temp_storage;
    (void)candidate_sort_temp_storage_bytes;
    if (k > 27 || unusable_rows_start > (1u << k) || !all_set({table, start_offset})) return cudaErrorInvalidValue;
    // start_offset spans n Fr = 2^(k+3) u32: 2^(k+2) slots keep the load <= 1/4
    return zk::lookup_table_build(CF(table), unusable_rows_start, reinterpret_cast<uint32_t*>(start_offset), k + 2,
                                  stream);
}

cudaError_t calc_m(void* m, void* table, void* input, void* sorted_index, void* start_offset, void* matched_index,
                   void* sorted_matched_index, void* candidate_sort_temp_storage,
                   uint32_t candidate_sort_temp_storage_bytes, uint32_t k, uint32_t unusable_rows_start,
                   cudaStream_t stream) {
    (void)sorted_index;
    (void)sorted_matched_index;
    (void)candidate_sort_temp_storage;
    (void)candidate_sort_temp_storage_bytes;
    if (k > 27 || unusable_rows_start > (1u << k) || !all_set({m, table, input, start_offset, matched_index}))
        return cudaErrorInvalidValue;
    return zk::lookup_count(F(m), CF(table), CF(input), 1u << k, unusable_rows_start,
                            reinterpret_cast<const uint32_t*>(start_offset), k + 2,
                            reinterpret_cast<uint32_t*>(matched_index), stream);
}

// ================================================================== Part 2

size_t zkp_msm_scratch_bytes(uint32_t n, int window_bits) { return msm_scratch_bytes(msm_make_plan(n, window_bits)); }

int zkp_msm_default_window(uint32_t n) { return msm_make_plan(n, 0).c; }

cudaError_t zkp_msm(void* out, const void* bases, const void* scalars, uint32_t n, int window_bits, void* scratch,
                    size_t scratch_bytes, cudaStream_t stream) {
    if (!out || (n && (!bases || !scalars || !scratch))) return cudaErrorInvalidValue;
    if (n > 0x7fffffffu) return cudaErrorInvalidValue;
    MsmPlan pl = msm_make_plan(n, window_bits);
    if (n && msm_scratch_bytes(pl) > scratch_bytes) return cudaErrorInvalidValue;
    MsmScratch sc = {};
    if (n) msm_layout(pl, scratch, &sc);
    return msm_run(reinterpret_cast<Jac*>(out), reinterpret_cast<const Aff*>(bases), CF(scalars), pl, sc, stream);
}

size_t zkp_msm_table_bytes(uint32_t nsrs, int window_bits) {
    return msm_table_points(nsrs, window_bits) * sizeof(Aff);
}

int zkp_msm_table_default_window(uint32_t n) { return msm_table_default_window(n); }

// table entries are addressed by 31-bit indices
static bool table_fits(uint32_t nsrs, int window_bits) {
    const size_t pts = msm_table_points(nsrs, window_bits);
    return pts > 0 && pts <= 0x80000000ull;
}

cudaError_t zkp_msm_table_build(void* table, const void* bases, uint32_t nsrs, int window_bits,
                                cudaStream_t stream) {
    if (nsrs && (!table || !bases)) return cudaErrorInvalidValue;
    if (!table_fits(nsrs ? nsrs : 1, window_bits)) return cudaErrorInvalidValue;
    return msm_table_build(reinterpret_cast<Aff*>(table), reinterpret_cast<const Aff*>(bases), nsrs, window_bits,
                           stream);
}

size_t zkp_msm_table_scratch_bytes(uint32_t n, int window_bits) {
    if (window_bits < 4 || window_bits > 22) return 0;
    return msm_scratch_bytes(msm_make_table_plan(n, window_bits, n ? n : 1));
}

cudaError_t zkp_msm_table(void* out, const void* table, uint32_t nsrs, int window_bits, const void* scalars,
                          uint32_t n, void* scratch, size_t scratch_bytes, cudaStream_t stream) {
    if (!out || (n && (!table || !scalars || !scratch))) return cudaErrorInvalidValue;
    if (n > nsrs || !table_fits(nsrs ? nsrs : 1, window_bits)) return cudaErrorInvalidValue;
    MsmPlan pl = msm_make_table_plan(n, window_bits, nsrs);
    if (n && msm_scratch_bytes(pl) > scratch_bytes) return cudaErrorInvalidValue;
    MsmScratch sc = {};
    if (n) msm_layout(pl, scratch, &sc);
    return msm_run(reinterpret_cast<Jac*>(out), reinterpret_cast<const Aff*>(table), CF(scalars), pl, sc, stream);
}

size_t zkp_msm_batch_scratch_bytes(const uint32_t* n, const int* window_bits, uint32_t count) {
    if (!n) return 0;
    return msm_batch_scratch_bytes(n, window_bits, count);
}

cudaError_t zkp_msm_batch(void* out, const void* bases, const void* scalars, const uint32_t* n,
                          const int* window_bits, uint32_t count, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    if (!out || !bases || !scalars || !n || !scratch) return cudaErrorInvalidValue;
    return msm_batch_run(reinterpret_cast<Jac*>(out), reinterpret_cast<const Aff*>(bases),
                         reinterpret_cast<const Fr* const*>(scalars), n, window_bits, count, scratch, scratch_bytes,
                         stream);
}

int zkp_msm_batch_table_default_window(const uint32_t* n, uint32_t count) {
    if (!n || count == 0) return msm_table_default_window(0);
    return msm_batch_table_default_window(n, count);
}

size_t zkp_msm_batch_table_scratch_bytes(const uint32_t* n, uint32_t count, uint32_t nsrs, int window_bits) {
    if (!n || nsrs == 0 || !table_fits(nsrs, window_bits)) return 0;
    return msm_batch_scratch_bytes(n, &window_bits, count, nsrs);
}

cudaError_t zkp_msm_batch_table(void* out, const void* table, uint32_t nsrs, int window_bits, const void* scalars,
                                const uint32_t* n, uint32_t count, void* scratch, size_t scratch_bytes,
                                cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    if (!out || !table || !scalars || !n || !scratch || nsrs == 0) return cudaErrorInvalidValue;
    if (!table_fits(nsrs, window_bits)) return cudaErrorInvalidValue;
    return msm_batch_run(reinterpret_cast<Jac*>(out), reinterpret_cast<const Aff*>(table),
                         reinterpret_cast<const Fr* const*>(scalars), n, &window_bits, count, scratch, scratch_bytes,
                         stream, nsrs);
}

cudaError_t zkp_ntt_batch(void* buf, void* tmp, const void* omegas, const void* scale, int log_n, uint32_t ncols,
                          size_t col_stride, int* result_in_tmp, cudaStream_t stream) {
    if (log_n < 1 || log_n > 28 || !buf || !omegas || !result_in_tmp || ncols == 0 || ncols > 65535)
        return cudaErrorInvalidValue;
    if (log_n > 12 && !tmp) return cudaErrorInvalidValue;
    bool in_tmp = false;
    ZK_CHECK(ntt_run(F(buf), F(tmp), CF(omegas), CF(scale), log_n, ncols, col_stride, &in_tmp, stream));
    *result_in_tmp = in_tmp ? 1 : 0;
    return cudaGetLastError();
}

int zkp_ntt_default_plan(int log_n, int* radices) {
    if (log_n < 1 || log_n > 28 || !radices) return 0;
    return ntt_plan(log_n, radices);
}

cudaError_t zkp_ntt_batch_plan(void* buf, void* tmp, const void* omegas, const void* scale, int log_n,
                               uint32_t ncols, size_t col_stride, const int* radices, int npasses,
                               int* result_in_tmp, cudaStream_t stream) {
    if (log_n < 3 || log_n > 28 || !buf || !omegas || !result_in_tmp || !radices || ncols == 0 || ncols > 65535)
        return cudaErrorInvalidValue;
    if (npasses < 1 || npasses > 4 || (npasses > 1 && !tmp)) return cudaErrorInvalidValue;
    int sum = 0;
    for (int i = 0; i < npasses; i++) {
        // every pass radix the pass kernels are built for at any size
        if (npasses > 1 && (radices[i] < 6 || radices[i] > 12)) return cudaErrorInvalidValue;
        if (npasses == 1 && radices[i] > 12) return cudaErrorInvalidValue;
        sum += radices[i];
    }
    if (sum != log_n) return cudaErrorInvalidValue;
    bool in_tmp = false;
    ZK_CHECK(ntt_run_plan(F(buf), F(tmp), CF(omegas), CF(scale), log_n, ncols, col_stride, radices, npasses, &in_tmp,
                          stream));
    *result_in_tmp = in_tmp ? 1 : 0;
    return cudaGetLastError();
}

cudaError_t zkp_powers(void* out, const void* base, const void* w, uint32_t n, cudaStream_t stream) {
    if (!out || !base || !w) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    return zk::geometric(F(out), CF(base), CF(w), n, stream);
}

#ifndef ZK_EXTEND_SECOND_RADIX
#define ZK_EXTEND_SECOND_RADIX 0  // 0: the even two-pass split
#endif

// passes of the extend phase: one pass up to 2^12, else two (first radix the
// larger half, at most 2^12), or with ZK_EXTEND_SECOND_RADIX a two-pass split
// whose second (fused) radix is that value.  The standalone NTT may split the
// same size into three passes; this phase is built on two.
static int extend_plan(int log_n, int* rad) {
    if (log_n <= 12) return ntt_plan(log_n, rad);
    rad[0] = (log_n + 1) / 2;
    rad[1] = log_n / 2;
    if (ZK_EXTEND_SECOND_RADIX > 0 && log_n - ZK_EXTEND_SECOND_RADIX >= 3 && log_n - ZK_EXTEND_SECOND_RADIX <= 12) {
        rad[1] = ZK_EXTEND_SECOND_RADIX;
        rad[0] = log_n - ZK_EXTEND_SECOND_RADIX;
    }
    return 2;
}

// the fused stage applies when the transform takes two passes whose second
// radix is 2^9..2^11 (two tiles of that radix fit in shared memory)
static bool extend_fused(int log_n, int* rad) {
    const int np = extend_plan(log_n, rad);
    return np == 2 && rad[1] >= 9 && rad[1] <= 11;
}

size_t zkp_coset_table_elems(int log_n, int ext_bits) {
    if (log_n < 1 || log_n > 28 || ext_bits < 0 || ext_bits > 6) return 0;
    int rad[4];
    const size_t n = (size_t)1 << log_n, E = (size_t)1 << ext_bits;
    return extend_fused(log_n, rad) ? E * n + E * ((size_t)1 << rad[1]) : E * n;
}

cudaError_t zkp_coset_twist_tables(void* twist, const void* shift, const void* w_ext, int log_n, int ext_bits,
                                   const void* tw, cudaStream_t stream) {
    if (log_n < 1 || log_n > 28 || ext_bits < 0 || ext_bits > 6 || !twist || !shift || !w_ext)
        return cudaErrorInvalidValue;
    int rad[4];
    const size_t n = (size_t)1 << log_n;
    if (extend_fused(log_n, rad)) {
        if (!tw) return cudaErrorInvalidValue;
        return zk::ntt_fused_tables(F(twist), F(twist) + (n << ext_bits), CF(tw), CF(shift), CF(w_ext), log_n, rad[1],
                                    ext_bits, stream);
    }
    const uint32_t chunk = 16;
    const uint32_t threads = (uint32_t)((n + chunk - 1) / chunk);
    dim3 grid((threads + 127) / 128, 1u << ext_bits);
    zk::twist_kernel<false><<<grid, 128, 0, stream>>>(F(twist), CF(shift), CF(w_ext), (uint32_t)n, chunk);
    return cudaGetLastError();
}

// Tables of zkp_extend_batch_tables, every factor as a (w, w') pair of
// fe_mul_shoup (two elements an entry), in elements:
//   [0, 2n) tw, [2n, 4n) tw_inv, [4n, 4n + 2) n^-1, then the coset tables of
//   zkp_coset_twist_tables (2 E n + 2 E 2^r for the fused stage, else 2 E n)
size_t zkp_extend_table_elems(int log_n, int ext_bits) {
    const size_t c = zkp_coset_table_elems(log_n, ext_bits);
    if (c == 0 || log_n > 24) return 0;
    return 4 * ((size_t)1 << log_n) + 2 + 2 * c;
}

cudaError_t zkp_extend_tables(void* tables, const void* tw, const void* tw_inv, const void* n_inv, const void* shift,
                              const void* w_ext, int log_n, int ext_bits, cudaStream_t stream) {
    if (zkp_extend_table_elems(log_n, ext_bits) == 0 || !tables || !tw || !tw_inv || !n_inv || !shift || !w_ext)
        return cudaErrorInvalidValue;
    const size_t n = (size_t)1 << log_n;
    Fr* t = F(tables);
    ZK_CHECK(zk::shoup_pairs(t, CF(tw), n, stream));
    ZK_CHECK(zk::shoup_pairs(t + 2 * n, CF(tw_inv), n, stream));
    ZK_CHECK(zk::shoup_pairs(t + 4 * n, CF(n_inv), 1, stream));
    Fr* twist = t + 4 * n + 2;
    int rad[4];
    if (extend_fused(log_n, rad))
        return zk::ntt_fused_tables(twist, twist + 2 * (n << ext_bits), CF(tw), CF(shift), CF(w_ext), log_n, rad[1],
                                    ext_bits, stream, true);
    const uint32_t chunk = 16;
    const uint32_t threads = (uint32_t)((n + chunk - 1) / chunk);
    dim3 grid((threads + 127) / 128, 1u << ext_bits);
    zk::twist_kernel<true><<<grid, 128, 0, stream>>>(twist, CF(shift), CF(w_ext), (uint32_t)n, chunk);
    return cudaGetLastError();
}

// the extended-domain phase over either table layout: Montgomery tables
// (pairs = 0) or (w, w') pairs; twist holds the coset tables (wtab then stab
// for the fused stage), offsets counted in entries of the layout
static cudaError_t extend_impl(void* ext_out, void* coeff_out, const void* lagrange_in, uint32_t ncols, int log_n,
                               int ext_bits, const Fr* tw_inv, const Fr* n_inv, const Fr* tw, const Fr* twist,
                               int pairs, void* stage_events, void* scratch, cudaStream_t stream) {
    cudaEvent_t* ev = reinterpret_cast<cudaEvent_t*>(stage_events);
#define ZK_MARK(i) \
    if (ev) ZK_CHECK(cudaEventRecord(ev[i], stream))
    ZK_MARK(0);
    if (log_n < 3 || log_n > 24 || ext_bits < 0 || ext_bits > 4 || ncols == 0 || ncols > 65535)
        return cudaErrorInvalidValue;
    if (!ext_out || !lagrange_in || !tw_inv || !n_inv || !tw || !twist || !scratch) return cudaErrorInvalidValue;
    const size_t n = (size_t)1 << log_n;
    const size_t ew = pairs ? 2 : 1;  // elements an entry
    const uint32_t E = 1u << ext_bits;
    int rad[4];
    const int np = extend_plan(log_n, rad);
    if (np > 2) return cudaErrorInvalidValue;
    if (coeff_out && extend_fused(log_n, rad)) {
        // 1. first inverse pass: lagrange -> coeff_out (intermediate, transformed in place next)
        NttPassArgs a = {};
        a.src = CF(lagrange_in);
        a.dst = F(coeff_out);
        a.tw = tw_inv;
        a.log_n = log_n;
        a.src_ys = n;
        a.dst_ys = n;
        a.pairs = pairs;
        ZK_CHECK(ntt_pass(a, rad[0], ncols, 1, stream));
        ZK_MARK(1);
        ZK_MARK(2);
        // 2. fused: last inverse pass + first pass of each coset's forward transform
        FusedExtendArgs f = {};
        f.src = F(coeff_out);
        f.coeff = F(coeff_out);
        f.sub = F(scratch);
        f.tw_inv = tw_inv;
        f.n_inv = n_inv;
        f.tw = tw;
        f.wtab = twist;
        f.stab = twist + ew * E * n;
        f.log_n = log_n;
        f.E = (int)E;
        f.src_ys = n;
        f.coeff_ys = n;
        f.sub_ys = n * E;
        f.pairs = pairs;
        ZK_CHECK(ntt_fused_extend(f, rad[1], ncols, stream));
        ZK_MARK(3);
        // 3. last pass of each coset's forward transform, interleaved output
        NttPassArgs b = {};
        b.tw = tw;
        b.log_n = log_n;
        b.log_p = rad[1];
        b.src = F(scratch);
        b.dst = F(ext_out);
        b.src_ys = n * E;
        b.src_zs = n;
        b.dst_ys = n * E;
        b.out_shift = ext_bits;
        b.out_off_z = 1;
        b.pairs = pairs;
        ZK_CHECK(ntt_pass(b, rad[0], ncols, E, stream));
        ZK_MARK(4);
        return cudaGetLastError();
    }
    Fr* scr = F(scratch);
    Fr* coeff = coeff_out ? F(coeff_out) : scr + (size_t)ncols * (E - 1) * n;
    // 1. inverse transform: lagrange -> (scratch) -> coefficients, scaled by n^-1
    {
        NttPassArgs a = {};
        a.tw = tw_inv;
        a.log_n = log_n;
        a.pairs = pairs;
        if (np == 1) {
            a.src = CF(lagrange_in);
            a.dst = coeff;
            a.scale = n_inv;
            a.src_ys = n;
            a.dst_ys = n;
            // single pass cannot run in place across buffers, so copy first
            if (a.src != a.dst)
                ZK_CHECK(cudaMemcpyAsync(coeff, lagrange_in, ncols * n * sizeof(Fr), cudaMemcpyDeviceToDevice, stream));
            a.src = coeff;
            ZK_MARK(1);
            ZK_CHECK(ntt_pass(a, rad[0], ncols, 1, stream));
        } else {
            a.src = CF(lagrange_in);
            a.dst = scr;
            a.log_p = 0;
            a.src_ys = n;
            a.dst_ys = n;
            ZK_CHECK(ntt_pass(a, rad[0], ncols, 1, stream));
            ZK_MARK(1);
            a.src = scr;
            a.dst = coeff;
            a.log_p = rad[0];
            a.scale = n_inv;
            ZK_CHECK(ntt_pass(a, rad[1], ncols, 1, stream));
        }
    }
    ZK_MARK(2);
    // 2. 2^e forward transforms of the twisted coefficients, interleaved output
    {
        NttPassArgs a = {};
        a.tw = tw;
        a.log_n = log_n;
        a.pairs = pairs;
        if (np == 1) {
            a.src = coeff;
            a.dst = F(ext_out);
            a.in_mul = twist;
            a.in_mul_zs = n;
            a.out_shift = ext_bits;
            a.out_off_z = 1;
            a.src_ys = n;
            a.dst_ys = n * E;
            ZK_MARK(3);
            ZK_CHECK(ntt_pass(a, rad[0], ncols, E, stream));
        } else {
            if (!coeff_out) return cudaErrorInvalidValue;  // scratch holds the sub-transforms
            a.src = coeff;
            a.dst = scr;
            a.in_mul = twist;
            a.in_mul_zs = n;
            a.src_ys = n;
            a.dst_ys = n * E;
            a.dst_zs = n;
            ZK_CHECK(ntt_pass(a, rad[0], ncols, E, stream));
            ZK_MARK(3);
            NttPassArgs b = {};
            b.tw = tw;
            b.log_n = log_n;
            b.pairs = pairs;
            b.log_p = rad[0];
            b.src = scr;
            b.dst = F(ext_out);
            b.src_ys = n * E;
            b.src_zs = n;
            b.dst_ys = n * E;
            b.out_shift = ext_bits;
            b.out_off_z = 1;
            ZK_CHECK(ntt_pass(b, rad[1], ncols, E, stream));
        }
    }
    ZK_MARK(4);
#undef ZK_MARK
    return cudaGetLastError();
}

cudaError_t zkp_extend_batch(void* ext_out, void* coeff_out, const void* lagrange_in, uint32_t ncols, int log_n,
                             int ext_bits, const void* tw_inv, const void* n_inv, const void* tw, const void* twist,
                             void* scratch, void* stage_events, cudaStream_t stream) {
    return extend_impl(ext_out, coeff_out, lagrange_in, ncols, log_n, ext_bits, CF(tw_inv), CF(n_inv), CF(tw),
                       CF(twist), 0, stage_events, scratch, stream);
}

cudaError_t zkp_extend_batch_tables(void* ext_out, void* coeff_out, const void* lagrange_in, uint32_t ncols,
                                    int log_n, int ext_bits, const void* tables, void* scratch, void* stage_events,
                                    cudaStream_t stream) {
    if (!tables || log_n < 3 || log_n > 24) return cudaErrorInvalidValue;
    const size_t n = (size_t)1 << log_n;
    const Fr* t = CF(tables);
    return extend_impl(ext_out, coeff_out, lagrange_in, ncols, log_n, ext_bits, t + 2 * n, t + 4 * n, t,
                       t + 4 * n + 2, 1, stage_events, scratch, stream);
}

cudaError_t zkp_batch_inverse(void* out, const void* in, const void* c, uint32_t n, int accumulate, void* scratch,
                              cudaStream_t stream) {
    if (n && (!out || !in)) return cudaErrorInvalidValue;
    return zk::batch_inverse(F(out), CF(in), CF(c), n, accumulate, F(scratch), scratch ? fr_scan_tmp_elems(n) : 0,
                             stream);
}

size_t zkp_scan_scratch_elems(uint32_t n) { return fr_scan_tmp_elems(n); }

uint32_t zkp_scan_timeouts(void) { return fr_scan_timeouts(); }

cudaError_t zkp_fr_to_mont(void* out, const void* in, uint32_t n, cudaStream_t stream) {
    if (n && (!out || !in)) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    zk::to_mont_kernel<<<(n + 255) / 256, 256, 0, stream>>>(F(out), CF(in), n);
    return cudaGetLastError();
}

cudaError_t zkp_g1_multiples(void* out, const void* k64, uint32_t n, cudaStream_t stream) {
    if (n && (!out || !k64)) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    zk::g1_multiples_kernel<<<(n + 127) / 128, 128, 0, stream>>>(reinterpret_cast<Aff*>(out),
                                                                 reinterpret_cast<const uint64_t*>(k64), n);
    return cudaGetLastError();
}

cudaError_t zkp_grand_product(void* out, const void* in, uint32_t n, const void* init, void* scratch,
                              cudaStream_t stream) {
    if (n && (!out || !in || !scratch)) return cudaErrorInvalidValue;
    return fr_scan_excl(F(out), CF(in), n, CF(init), 1, F(scratch), stream);
}

cudaError_t zkp_grand_sum(void* out, const void* in, uint32_t n, const void* init, void* scratch,
                          cudaStream_t stream) {
    if (n && (!out || !in || !scratch)) return cudaErrorInvalidValue;
    return fr_scan_excl(F(out), CF(in), n, CF(init), 0, F(scratch), stream);
}

cudaError_t zkp_permutation_z(void* z, const void* cols, const void* sigmas, int ncols, const void* beta,
                              const void* gamma, const void* dbeta, const void* omegas, const void* init, uint32_t n,
                              void* scratch, cudaStream_t stream) {
    if (ncols <= 0 || !z || !cols || !sigmas || !beta || !gamma || !dbeta || !omegas || !scratch)
        return cudaErrorInvalidValue;
    return permutation_chunk_z(F(z), reinterpret_cast<const Fr* const*>(cols),
                               reinterpret_cast<const Fr* const*>(sigmas), ncols, CF(beta), CF(gamma), CF(dbeta),
                               CF(omegas), CF(init), n, F(scratch), stream);
}

cudaError_t zkp_shuffle_z(void* z, const void* inputs, const void* tables, const void* betas, int groups, uint32_t n,
                          void* scratch, cudaStream_t stream) {
    if (groups <= 0 || !z || !inputs || !tables || !betas || !scratch) return cudaErrorInvalidValue;
    return shuffle_z(F(z), reinterpret_cast<const Fr* const*>(inputs), reinterpret_cast<const Fr* const*>(tables),
                     CF(betas), groups, n, F(scratch), F(scratch) + n, stream);
}

}  // extern "C"

// ================================================================== Part 3: calibration

namespace zk {
// Each thread runs 4 independent chains of dependent Montgomery products,
// `iters` steps each; measures the sustainable Fr multiplication rate that
// bounds the integer-pipe kernels (NTT butterflies, MSM point additions).
__global__ void __launch_bounds__(256) mont_rate_kernel(Fr* out, uint32_t iters) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    Fr a = fe_one<FrCfg>(), b = fe_one<FrCfg>(), c = fe_one<FrCfg>(), d = fe_one<FrCfg>();
    a.v[0] ^= t;
    b.v[1] ^= t;
    c.v[2] ^= t;
    d.v[3] ^= t;
    Fr m = a;
    m.v[5] ^= 0x1234u;
    for (uint32_t i = 0; i < iters; i++) {
        a = fe_mul<FrCfg>(a, m);
        b = fe_mul<FrCfg>(b, m);
        c = fe_mul<FrCfg>(c, m);
        d = fe_mul<FrCfg>(d, m);
    }
    Fr s = fe_add<FrCfg>(fe_add<FrCfg>(a, b), fe_add<FrCfg>(c, d));
    if (fe_is_zero<FrCfg>(s)) st_elem<FrCfg>(out, s);
}

// The same for products by a known factor (fe_mul_shoup), the form of every
// product of the extend-phase kernels over pair tables; wtab[0], wtab[1] is a
// (w, w') pair.
__global__ void __launch_bounds__(256) shoup_rate_kernel(Fr* out, const Fr* wtab, uint32_t iters) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    Fr a = fe_one<FrCfg>(), b = fe_one<FrCfg>(), c = fe_one<FrCfg>(), d = fe_one<FrCfg>();
    a.v[0] ^= t;
    b.v[1] ^= t;
    c.v[2] ^= t;
    d.v[3] ^= t;
    const Fr w = ld_elem<FrCfg>(wtab), wp = ld_elem<FrCfg>(wtab + 1);
    for (uint32_t i = 0; i < iters; i++) {
        a = fe_mul_shoup<FrCfg>(a, w, wp);
        b = fe_mul_shoup<FrCfg>(b, w, wp);
        c = fe_mul_shoup<FrCfg>(c, w, wp);
        d = fe_mul_shoup<FrCfg>(d, w, wp);
    }
    Fr s = fe_add<FrCfg>(fe_add<FrCfg>(a, b), fe_add<FrCfg>(c, d));
    if (fe_is_zero<FrCfg>(s)) st_elem<FrCfg>(out, s);
}
}  // namespace zk

extern "C" cudaError_t zkp_calib_mont_rate(void* out, uint32_t blocks, uint32_t iters, cudaStream_t stream) {
    if (!out || blocks == 0) return cudaErrorInvalidValue;
    zk::mont_rate_kernel<<<blocks, 256, 0, stream>>>(F(out), iters);
    return cudaGetLastError();
}

// out: one element of scratch (written only when a sum is zero); pair: a
// (w, w') pair on the device
extern "C" cudaError_t zkp_calib_shoup_rate(void* out, const void* pair, uint32_t blocks, uint32_t iters,
                                            cudaStream_t stream) {
    if (!out || !pair || blocks == 0) return cudaErrorInvalidValue;
    zk::shoup_rate_kernel<<<blocks, 256, 0, stream>>>(F(out), CF(pair), iters);
    return cudaGetLastError();
}
