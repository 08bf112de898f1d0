// Internal C++ interface between the kernels and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include "field.cuh"
#include "curve.cuh"

namespace zk {

// ------------------------------------------------------------------ NTT
struct NttPassArgs {
    const Fr* src;
    Fr* dst;
    const Fr* tw;        // natural table w^i, i < 2^log_n
    int log_n;
    int log_p;           // log2 of the product of the radices of earlier passes
    const Fr* in_mul;    // optional multiplier per natural input position (first pass only)
    const Fr* scale;     // optional multiplier of every output (last pass only)
    int out_shift;       // output index = (pos << out_shift) + blockIdx.z * out_off_z
    size_t out_off_z;
    size_t src_ys, dst_ys;  // per-column strides (blockIdx.y), elements
    size_t src_zs, dst_zs;  // per-sub-transform strides (blockIdx.z), elements
    size_t in_mul_zs;
    int pairs;           // tw, in_mul and scale hold (w, w') pairs (two elements an entry)
};

cudaError_t ntt_pass(const NttPassArgs& a, int log_r, unsigned ny, unsigned nz, cudaStream_t s);

// fused last inverse pass + first pass of every coset's forward transform
struct FusedExtendArgs {
    const Fr* src;     // inverse-transform intermediate (may alias coeff)
    Fr* coeff;         // coefficients, natural order
    Fr* sub;           // per-coset first-pass outputs, E * n per column
    const Fr* tw_inv;  // w^-i, n entries
    const Fr* n_inv;
    const Fr* tw;      // w^i, n entries
    const Fr* wtab;    // E * n
    const Fr* stab;    // E * 2^log_r
    int log_n, E;
    size_t src_ys, coeff_ys, sub_ys;
    int pairs;         // every table holds (w, w') pairs (two elements an entry)
};
cudaError_t ntt_fused_extend(const FusedExtendArgs& a, int log_r, unsigned ncols, cudaStream_t s);
cudaError_t ntt_fused_tables(Fr* wtab, Fr* stab, const Fr* tw, const Fr* shift, const Fr* w_ext, int log_n, int log_r,
                             int ext_bits, cudaStream_t s, bool pairs = false);
// out[2i], out[2i+1] = (w, w') of the Montgomery-form factors in[i], i < n
cudaError_t shoup_pairs(Fr* out, const Fr* in, size_t n, cudaStream_t s);
int ntt_plan(int log_n, int radices[4]);
// Full transform of ncols columns (stride col_stride elements) by the twiddle
// table tw; result in buf or tmp (*result_in_tmp), multiplied by *scale if given.
cudaError_t ntt_run(Fr* buf, Fr* tmp, const Fr* tw, const Fr* scale, int log_n, unsigned ncols,
                    size_t col_stride, bool* result_in_tmp, cudaStream_t s);
// the same with the pass radices given (np passes, sum log_n)
cudaError_t ntt_run_plan(Fr* buf, Fr* tmp, const Fr* tw, const Fr* scale, int log_n, unsigned ncols,
                         size_t col_stride, const int* rad, int np, bool* result_in_tmp, cudaStream_t s);
cudaError_t expand_powers(Fr* buf, uint32_t n, cudaStream_t s);
cudaError_t geometric(Fr* out, const Fr* base, const Fr* w, uint32_t n, cudaStream_t s);

// ------------------------------------------------------------------ MSM
struct MsmPlan {
    int c;          // window bits (signed digits in [-(2^(c-1)-1), 2^(c-1)])
    int W;          // windows (digits per scalar)
    uint32_t B;     // buckets per window, 2^(c-1)
    uint32_t NB;    // Wb * B
    uint32_t L;     // sorted entries per accumulation thread
    uint32_t nacc;  // accumulation threads
    uint32_t seg;   // buckets per reduction segment
    uint32_t G;     // reduction segments per bucket set
    uint32_t n;
    int glv;        // 1: scalars split k = k1 + k2 lambda over the bases and their endomorphism images
    int Wb;         // bucket sets: W, or 1 over a table of pre-multiplied bases
    uint32_t nsrs;  // table plans: points per window of the table (0: no table)
};

struct MsmScratch {
    uint32_t* count;     // NB
    uint32_t* offset;    // NB + 1
    uint32_t* scan_tmp;  // scan_tmp_words(NB)
    uint32_t* entries;   // n * W
    uint32_t* part_key;  // 2 * nacc + msm_merge_extra(nacc)
    Xyzz* part_pt;       // 2 * nacc + msm_merge_extra(nacc)
    Xyzz* buckets;       // NB
    Xyzz* segsum;        // Wb * G
    Xyzz* winsum;        // Wb
    Aff* phi;            // n endomorphism images of the bases (GLV plans without a table), else null
};

MsmPlan msm_make_plan(uint32_t n, int c, bool glv = true);
// plan over a table of pre-multiplied bases (msm_table_*): all windows share
// one bucket set; the table holds nsrs >= n points per window
MsmPlan msm_make_table_plan(uint32_t n, int c, uint32_t nsrs);
// window bits the library picks for an MSM of n points over a table
int msm_table_default_window(uint32_t n);
int msm_batch_table_default_window(const uint32_t* n, uint32_t count);
// Table of pre-multiplied bases: for window j < W (W = ceil(128 / c)) and
// i < nsrs, entry j 2 nsrs + i is [2^(c j)] base_i and entry
// j 2 nsrs + nsrs + i its endomorphism image, as affine points.
size_t msm_table_points(uint32_t nsrs, int c);
cudaError_t msm_table_build(Aff* table, const Aff* bases, uint32_t nsrs, int c, cudaStream_t st);
// sorted entries (nonzero digits at most) of a plan: n W, or 2 n W with GLV
inline size_t msm_entry_count(const MsmPlan& p) { return (size_t)p.n * p.W * (p.glv ? 2 : 1); }
size_t msm_u32_words(const MsmPlan& p);     // count + offset + scan tmp + entries + part keys
size_t msm_point_count(const MsmPlan& p);   // partial points + buckets + segment and window sums
size_t msm_scratch_bytes(const MsmPlan& p); // one contiguous scratch area (both of the above)
void msm_layout(const MsmPlan& p, void* base, MsmScratch* s);
void msm_layout_split(const MsmPlan& p, uint32_t* words, Xyzz* points, MsmScratch* s);
// places the plan's buffers (largest first, 256-byte aligned) into the first
// of up to 8 caller arenas with room, the window sums only into arena
// winsum_arena when that is not negative; false when they do not fit
bool msm_layout_arenas(const MsmPlan& p, void* const* arena, const size_t* arena_bytes, int n_arenas,
                       MsmScratch* s, int winsum_arena = -1);
// sum_i [scalars_i] bases_i written as a Jacobian point at out; scalars in
// Montgomery form; no allocation, no host synchronisation.
// With park_note set (8-byte aligned), the final combination is left out: the
// window sums stay in scratch and a 24-byte note at park_note records where;
// msm_collect finishes such MSMs.
cudaError_t msm_run(Jac* out, const Aff* bases, const Fr* scalars, const MsmPlan& p, const MsmScratch& s,
                    cudaStream_t st, void* park_note = nullptr);
// final combinations of count parked MSMs: regions[i] + note_off holds the
// note, the Jacobian result goes to regions[i] (device array of pointers)
cudaError_t msm_collect(char* const* regions, uint32_t count, uint32_t note_off, cudaStream_t st);

size_t msm_merge_extra(uint32_t nacc);  // merge-level items after the 2 * nacc partials
// part_key / part_pt hold 2 * nacc + msm_merge_extra(nacc) items
// entry points below nbase index bases, the others phi (GLV images)
cudaError_t msm_accumulate_merge(const uint32_t* entries, const uint32_t* offset, uint32_t NB, const Aff* bases,
                                 const Aff* phi, uint32_t nbase, uint32_t L, uint32_t nacc, Xyzz* buckets,
                                 uint32_t* part_key, Xyzz* part_pt, cudaStream_t st);
// phi[i] = (beta x_i, y_i) for i < n
cudaError_t msm_phi(const Aff* bases, uint32_t n, Aff* phi, cudaStream_t st);

// nsrs > 0: bases is a table of pre-multiplied bases (msm_table_build with
// nsrs points and width c[0]) and every MSM runs over it with that width
size_t msm_batch_scratch_bytes(const uint32_t* n, const int* c, uint32_t count, uint32_t nsrs = 0);
cudaError_t msm_batch_run(Jac* out, const Aff* bases, const Fr* const* scalars, const uint32_t* n, const int* c,
                          uint32_t count, void* scratch, size_t scratch_bytes, cudaStream_t st, uint32_t nsrs = 0);

// ------------------------------------------------------------------ scans
size_t scan_tmp_words(uint32_t n);
// exclusive prefix sum of n u32 values; out[n] = total
cudaError_t scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s);


// ------------------------------------------------------------------ elementwise (eval_h)
cudaError_t field_op(Fr* res, const Fr* l, int l_rot, const Fr* l_c, const Fr* r, int r_rot, const Fr* r_c,
                     uint32_t n, int op, cudaStream_t s);
cudaError_t field_op_batch_mul_sum(Fr* res, Fr* const* v, const int* rot, int n_v, uint32_t n, cudaStream_t s);
cudaError_t extended_prepare(Fr* s, const Fr* coset_powers, uint32_t cpn, uint32_t size, uint32_t ext_size,
                             int to_coset, cudaStream_t st);
cudaError_t permutation_eval_h_p1(Fr* res, const Fr* first_set, const Fr* last_set, const Fr* l0,
                                  const Fr* l_last, const Fr* y, uint32_t n, cudaStream_t s);
cudaError_t permutation_eval_h_p2(Fr* res, const Fr* const* set, const Fr* l0, const Fr* y, int n_set, int rot,
                                  uint32_t n, cudaStream_t s);
cudaError_t permutation_eval_h_l(Fr* res, const Fr* beta, const Fr* gamma, const Fr* p, uint32_t n,
                                 cudaStream_t s);
cudaError_t lookup_eval_h(Fr* res, const Fr* input, const Fr* table, const Fr* permuted_input,
                          const Fr* permuted_table, const Fr* z, const Fr* l0, const Fr* l_last,
                          const Fr* l_active_row, const Fr* y, const Fr* beta, const Fr* gamma, int rot, uint32_t n,
                          cudaStream_t s);
cudaError_t logup_eval_h(Fr* res, const Fr* input_product, const Fr* input_product_sum, const Fr* table,
                         const Fr* multiplicity, const Fr* z_first, const Fr* z_last, const Fr* l0,
                         const Fr* l_last, const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s);
cudaError_t logup_eval_h_extra_inputs(Fr* res, const Fr* input_product, const Fr* input_product_sum, const Fr* z,
                                      const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s);
cudaError_t logup_eval_h_inputs_product_sum(Fr* product, Fr* product_sum, const Fr* const* set, int n_set,
                                            uint32_t n, cudaStream_t s);
cudaError_t shuffle_eval_h(Fr* res, const Fr* input, const Fr* table, const Fr* z, const Fr* l0, const Fr* l_last,
                           const Fr* l_active_row, const Fr* y, int rot, uint32_t n, cudaStream_t s);
cudaError_t shuffle_eval_h_v2(Fr* res, const Fr* const* inputs, const Fr* const* tables, const Fr* betas,
                              int group_len, const Fr* z, const Fr* l0, const Fr* l_last, const Fr* l_active_row,
                              const Fr* y, int rot, uint32_t n, cudaStream_t s);
cudaError_t field_mul_zip(Fr* buf, const Fr* coeff, uint32_t coeff_n, uint32_t n, cudaStream_t s);
cudaError_t field_sum(Fr* res, Fr* const* v, Fr* const* v_c, const int* v_rot, const Fr* omegas, int v_n,
                      uint32_t n, cudaStream_t s);
cudaError_t shplonk_h_x_merge(Fr* res, const Fr* v, const Fr* values, const Fr* omegas, const Fr* diff_points,
                              int diff_points_n, uint32_t n, cudaStream_t s);


// ------------------------------------------------------------------ Fr scans
// scratch (may be null) of at least batch_inv_scratch_elems(n) elements
// selects the three-phase form with a single field inversion
size_t batch_inv_scratch_elems(uint32_t n);
cudaError_t batch_inverse(Fr* out, const Fr* in, const Fr* c, uint32_t n, int accumulate, Fr* scratch,
                          size_t scratch_elems, cudaStream_t s);
cudaError_t div_by_point_diffs(Fr* values, const Fr* omegas, const Fr* points, int np, uint32_t n, Fr* scratch,
                               size_t scratch_elems, cudaStream_t s);
size_t fr_scan_tmp_elems(uint32_t n);
uint32_t fr_scan_timeouts();
cudaError_t fr_scan_excl(Fr* out, const Fr* in, uint32_t n, const Fr* init, int op, Fr* tmp, cudaStream_t s);
cudaError_t logup_z_scan(Fr* z, Fr* last_z, int last_index, uint32_t n, Fr* tmp, cudaStream_t s);
cudaError_t logup_z_compose(Fr* z, const Fr* sum, const Fr* table, const Fr* m, const Fr* beta, Fr* last_z,
                            int last_index, uint32_t n, Fr* tmp, cudaStream_t s);
cudaError_t permutation_chunk_z(Fr* z, const Fr* const* cols, const Fr* const* sig, int ncols, const Fr* beta,
                                const Fr* gamma, const Fr* dbeta, const Fr* omegas, const Fr* init, uint32_t n,
                                Fr* tmp, cudaStream_t s);
cudaError_t shuffle_z(Fr* z, const Fr* const* inputs, const Fr* const* tables, const Fr* betas, int groups,
                      uint32_t n, Fr* num_tmp, Fr* tmp, cudaStream_t s);

// ------------------------------------------------------------------ lookup / poly
cudaError_t lookup_table_build(const Fr* table, uint32_t usable, uint32_t* slots, uint32_t log_slots,
                               cudaStream_t s);
cudaError_t lookup_count(Fr* m, const Fr* table, const Fr* input, uint32_t n, uint32_t usable, const uint32_t* slots,
                         uint32_t log_slots, uint32_t* cnt, cudaStream_t s);
cudaError_t poly_eval(const Fr* p, Fr* res, const Fr* x_table, uint32_t n, cudaStream_t s);

}  // namespace zk
