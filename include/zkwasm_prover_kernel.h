/*
 * C ABI of the B200 (sm_100a) KZG proving kernels for BN254.
 *
 * Part 1 is a drop-in for the reference's static library
 * `zkwasm_prover_kernel` (build.rs:5-10): the same 27 symbols with the
 * signatures the Rust FFI declares in src/cuda/bn254_c.rs:4-309.  Conventions,
 * as in the reference:
 *   - every pointer is a device pointer; Fr / Fq elements are 32 bytes
 *     (4 x u64 little-endian, Montgomery form, R = 2^256); G1 affine points
 *     are 64 bytes (x, y; identity (0, 0)); G1 Jacobian points 96 bytes
 *     (X, Y, Z; identity Z = 0);
 *   - `T**` arguments are device arrays of device pointers;
 *   - the return value is cudaGetLastError() after enqueueing (asynchronous);
 *   - entry points without a stream argument run on the legacy default stream.
 * Rotations are taken modulo n for either sign.  None of these functions
 * allocates device memory or blocks the host (the reference's msm does both:
 * cuda/msm.cu:384-418).
 *
 * Part 2 adds batched, allocation-free entry points (prefix zkp_) that the
 * Rust host can call for whole phases; their scratch memory is supplied by the
 * caller and sized by the matching *_scratch_bytes query.
 */
#ifndef ZKWASM_PROVER_KERNEL_H
#define ZKWASM_PROVER_KERNEL_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================
 * Part 1: reference-compatible symbols
 * ==================================================================== */

/* src/cuda/bn254_c.rs:6-16, cuda/bn254.cu:1357-1428.  Natural-order NTT of
 * 2^array_log elements by the twiddle table `omega` built by
 * expand_omega_buffer; scaled by *n_inv when n_inv is non-null (inverse
 * transform).  The result is in `buf` if *(bool*)swap is false on return,
 * else in `tmp`; *swap is written synchronously.  `pq` and `max_deg` are
 * accepted and unused. */
cudaError_t ntt(void *buf, void *tmp, void *pq, void *omega, void *n_inv, int array_log, int max_deg, void *swap,
                cudaStream_t stream);

/* src/cuda/bn254_c.rs:18-29, cuda/bn254.cu:1269-1286.  res[i] = L op R with
 * L = l[(i+l_rot) mod size] (* l_c[0]) or l_c[0], R likewise;
 * op 0 add, 1 mul, 2 copy L, 3 sub. */
cudaError_t field_op(void *res, void *l, int l_rot, void *l_c, void *r, int r_rot, void *r_c, int size, int op,
                     cudaStream_t stream);

/* src/cuda/bn254_c.rs:31-39, cuda/bn254.cu:1232-1253.  to_coset == 0: zero
 * s[size..extended_size) and multiply s[i] (i < size) by
 * coset_powers[i mod coset_powers_n - 1] when i mod coset_powers_n != 0;
 * to_coset != 0: the same multiply over i < extended_size. */
cudaError_t extended_prepare(void *s, void *coset_powers, int coset_powers_n, int size, int extended_size,
                             int to_coset, cudaStream_t stream);

/* src/cuda/bn254_c.rs:41-49, cuda/bn254.cu:1288-1303 (default stream) */
cudaError_t permutation_eval_h_p1(void *res, void *first_set, void *last_set, void *l0, void *l_last, void *y,
                                  int n);

/* src/cuda/bn254_c.rs:51-60, cuda/bn254.cu:1305-1319 (default stream) */
cudaError_t permutation_eval_h_p2(void *res, void *set, void *l0, void *l_last, void *y, int n_set, int rot, int n);

/* src/cuda/bn254_c.rs:62-69, cuda/bn254.cu:1321-1331 */
cudaError_t permutation_eval_h_l(void *res, void *beta, void *gamma, void *p, int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:71-79, cuda/bn254.cu:1217-1230 (default stream) */
cudaError_t field_sum(void *res, void *v, void *v_c, void *v_rot, void *omegas, int v_n, int n);

/* src/cuda/bn254_c.rs:81-88, cuda/bn254.cu:1255-1267.
 * v = [coeff0, a00, a01, NULL, coeff1, a10, NULL, ...] (v_n entries),
 * rot = one rotation per column entry; res[i] += sum_t coeff_t prod_j a_tj[i+rot]. */
cudaError_t field_op_batch_mul_sum(void *res, void *v, void *rot, int v_n, int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:90-106, cuda/bn254.cu:1430-1456 */
cudaError_t lookup_eval_h(void *res, void *input, void *table, void *permuted_input, void *permuted_table, void *z,
                          void *l0, void *l_last, void *l_active_row, void *y, void *beta, void *gamma, int rot,
                          int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:108-123, cuda/bn254.cu:1480-1504 */
cudaError_t logup_eval_h(void *res, void *input_product, void *input_product_sum, void *table, void *multiplicity,
                         void *z_first, void *z_last, void *l0, void *l_last, void *l_active_row, void *y, int rot,
                         int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:125-135, cuda/bn254.cu:1506-1522 */
cudaError_t logup_eval_h_extra_inputs(void *res, void *input_product, void *input_product_sum, void *z,
                                      void *l_active_row, void *y, int rot, int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:137-147, cuda/bn254.cu:1524-1541 */
cudaError_t logup_eval_h_z_set(void *res, void *set, void *l0, void *l_last, void *y, int n_set, int rot, int n,
                               cudaStream_t stream);

/* src/cuda/bn254_c.rs:149-157, cuda/bn254.cu:1914-1934.
 * sum[i] = (init ? sum[i] : 0) + 1 / (input[i] + beta[0]).  `temp` is unused. */
cudaError_t logup_sum_input_inv(void *sum, void *input, void *temp, void *beta, int init, int n,
                                cudaStream_t stream);

/* src/cuda/bn254_c.rs:159-166, cuda/bn254.cu:1995-2010 */
cudaError_t logup_eval_h_inputs_product_sum(void *product, void *product_sum, void *sets, int n_set, int n,
                                            cudaStream_t stream);

/* src/cuda/bn254_c.rs:168-179, cuda/bn254.cu:1458-1478 (default stream) */
cudaError_t shuffle_eval_h(void *res, void *input, void *table, void *z, void *l0, void *l_last, void *l_active_row,
                           void *y, int rot, int n);

/* src/cuda/bn254_c.rs:181-194, cuda/bn254.cu:1543-1566 (default stream) */
cudaError_t shuffle_eval_h_v2(void *res, void *inputs, void *tables, void *betas, int group_len, void *z, void *l0,
                              void *l_last, void *l_active_row, void *y, int rot, int n);

/* src/cuda/bn254_c.rs:196, cuda/bn254.cu:1333-1355 (default stream).
 * buf[0] = 1 and buf[1] = w are written by the caller; fills buf[i] = w^i for
 * i < 2^n.  The table is natural order whatever may_bit_reversed says; ntt()
 * is its only consumer besides the shplonk kernels, which need natural order. */
cudaError_t expand_omega_buffer(void *buf, int n, int may_bit_reversed);

/* src/cuda/bn254_c.rs:198, cuda/bn254.cu:1568-1578 (default stream) */
cudaError_t field_mul_zip(void *buf, void *coeff, int coeff_n, int n);

/* src/cuda/bn254_c.rs:200-206, cuda/bn254.cu:1608-1634.  x = table of
 * x^(2^d), d < log2 n; res (n elements) is workspace and res[0] = p(x). */
cudaError_t poly_eval(void *p, void *res, void *x, int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:208-216, cuda/bn254.cu:1580-1592 (default stream) */
cudaError_t shplonk_h_x_merge(void *res, void *v, void *values, void *omegas, void *diff_points, int diff_points_n,
                              int n);

/* src/cuda/bn254_c.rs:218-224, cuda/bn254.cu:1594-1606 (default stream);
 * values[i] /= prod_j (omegas[i] - points[j]) by batch inversion. */
cudaError_t shplonk_h_x_div_points(void *values, void *omegas, void *points, int points_n, int n);

/* src/cuda/bn254_c.rs:226-236, cuda/bn254.cu:1968-1993.
 * z = *last_z + exclusive prefix sum of input[i] - multiplicity[i]/(table[i]+beta);
 * then *last_z = z[last_z_index].  `table` is used as scratch (as in the
 * reference); `input` is not modified. */
cudaError_t eval_logup_z_compose(void *z, void *input, void *table, void *multiplicity, void *beta, void *last_z,
                                 int last_z_index, int n, cudaStream_t stream);

/* src/cuda/bn254_c.rs:238-246, cuda/bn254.cu:1936-1966.  z = *last_z +
 * exclusive prefix sum of z (in place); *last_z = z[last_z_index]; `table` is
 * scratch (n/2048 + 2 elements), `input` is unused. */
cudaError_t eval_logup_z_pure(void *z, void *input, void *table, void *last_z, int last_z_index, int n,
                              cudaStream_t stream);

/* src/cuda/bn254_c.rs:248-259, cuda/msm.cu:434-467.  buckets is the device
 * array of batch_size pointers to the per-MSM regions msm() ran in
 * (src/cuda/msm.rs:387-420); one launch runs the final window combination of
 * every MSM side by side and writes each Jacobian result where the reference
 * does, element 0 of its region.  Must follow the msm() calls in stream order
 * (the reference host synchronises their streams first).  Returns pending
 * errors of earlier launches, as the reference does.  The other arguments are
 * accepted and unused. */
cudaError_t batch_msm_collect(void *remain_indices, void *remain_acc, void *next_remain_indices,
                              void *next_remain_acc, void *buckets, uint32_t workers, uint32_t windows,
                              uint32_t window_bits, uint32_t batch_size, cudaStream_t stream);

/* src/cuda/bn254_c.rs:261-279, cuda/msm.cu:350-432.  Computes
 * sum_i [s_i] p_i for array_len affine bases p and Montgomery-form scalars s
 * up to the per-window sums, which stay in the region with a note of where
 * they are; batch_msm_collect then writes the Jacobian sum to res[0] (96
 * bytes), as in the reference.  res must span the reference's per-MSM region
 * of (windows << window_bits) + 2 * workers Jacobian points and sort_buf
 * 3 * array_len * windows u32 (the sizes src/cuda/msm.rs:297-317 allocates);
 * both are used as scratch.  The other index buffers, threads, workers, the
 * sort-storage size and skip_zero are accepted and unused.  Never blocks the
 * host. */
cudaError_t msm(void *res, void *p, void *s, void *indices_buf0, void *indices_buf1, void *indices_buf2,
                void *indices_buf3, void *sort_buf, void *indices_buf, int array_len, int windows, int window_bits,
                int threads, int workers, int prepared_sort_indices_temp_storage_bytes, int skip_zero,
                cudaStream_t stream);

/* src/cuda/bn254_c.rs:281-293, cuda/bn254.cu:1863-1912.  Builds a hash index
 * of the table's usable rows in start_offset (2^(k+3) u32 available, as the
 * reference allocates n Fr). Other buffers unused. */
cudaError_t prepare_table_lookup(void *table, void *table_lowest_u32, void *sorted_table_lowest_u32, void *index,
                                 void *sorted_index, void *start_offset, void *candidate_sort_temp_storage,
                                 uint32_t candidate_sort_temp_storage_bytes, uint32_t k,
                                 uint32_t unusable_rows_start, cudaStream_t stream);

/* src/cuda/bn254_c.rs:295-308, cuda/bn254.cu:1796-1861.  m[row] += number of
 * usable input rows equal to table[row], crediting the largest usable row
 * among equal table values; matched_index holds the per-row counts. */
cudaError_t calc_m(void *m, void *table, void *input, void *sorted_index, void *start_offset, void *matched_index,
                   void *sorted_matched_index, void *candidate_sort_temp_storage,
                   uint32_t candidate_sort_temp_storage_bytes, uint32_t k, uint32_t unusable_rows_start,
                   cudaStream_t stream);

/* ======================================================================
 * Part 2: batched, allocation-free entry points
 * ==================================================================== */

/* Scratch bytes zkp_msm needs for n points with window_bits (0 = automatic). */
size_t zkp_msm_scratch_bytes(uint32_t n, int window_bits);

/* Window width zkp_msm picks for n points when window_bits is 0. */
int zkp_msm_default_window(uint32_t n);

/* One MSM: out (96-byte Jacobian) = sum_i [scalars_i] bases_i.  Replaces the
 * msm + batch_msm_collect pair (src/cuda/msm.rs:239-455) without host
 * synchronisation; capturable in a CUDA graph. */
cudaError_t zkp_msm(void *out, const void *bases, const void *scalars, uint32_t n, int window_bits, void *scratch,
                    size_t scratch_bytes, cudaStream_t stream);

/* Tables of pre-multiplied bases for MSMs over a resident base array (the
 * SRS of a proving key; the reference host passes the same device bases to
 * every msm call, src/cuda/msm.rs:256-455).  A table for window_bits c
 * (4..22) holds W = ceil(128 / c) windows of 2 nsrs affine points:
 * [2^(c j)] bases_i at j 2 nsrs + i and its endomorphism image at
 * j 2 nsrs + nsrs + i.  zkp_msm_table_bytes is 0 for an unsupported width. */
size_t zkp_msm_table_bytes(uint32_t nsrs, int window_bits);

/* Window width the library picks for an MSM of n points over a table. */
int zkp_msm_table_default_window(uint32_t n);

/* Fills a table of zkp_msm_table_bytes(nsrs, window_bits) bytes from nsrs
 * affine bases (Montgomery form, the identity as (0, 0)). */
cudaError_t zkp_msm_table_build(void *table, const void *bases, uint32_t nsrs, int window_bits,
                                cudaStream_t stream);

/* Scratch bytes of zkp_msm_table for n points (0 for an unsupported width). */
size_t zkp_msm_table_scratch_bytes(uint32_t n, int window_bits);

/* out (96-byte Jacobian) = sum_{i < n} [scalars_i] bases_i over a table built
 * with the same nsrs and window_bits (n <= nsrs).  All windows share one
 * bucket set: no doublings between windows and one bucket reduction.  No
 * allocation, no host synchronisation. */
cudaError_t zkp_msm_table(void *out, const void *table, uint32_t nsrs, int window_bits, const void *scalars,
                          uint32_t n, void *scratch, size_t scratch_bytes, cudaStream_t stream);

/* Scratch bytes of zkp_msm_batch for `count` MSMs of n[i] points with window
 * widths window_bits[i] (host arrays; window_bits NULL or 0 entries pick the
 * default width for each size). */
size_t zkp_msm_batch_scratch_bytes(const uint32_t *n, const int *window_bits, uint32_t count);

/* A batch of MSMs over one base array in one pipeline (replaces the per-column
 * msm loop and batch_msm_collect of src/cuda/msm.rs:256-455):
 * out[i] (96-byte Jacobian, contiguous) = sum_{j < n[i]} [scalars[i][j]] bases[j],
 * scalars a device array of `count` device pointers, n and window_bits host
 * arrays.  The per-MSM descriptors travel as kernel parameters (one small
 * launch per 64 MSMs), so the call is capturable in a CUDA graph; no
 * allocation and no host synchronisation. */
cudaError_t zkp_msm_batch(void *out, const void *bases, const void *scalars, const uint32_t *n,
                          const int *window_bits, uint32_t count, void *scratch, size_t scratch_bytes,
                          cudaStream_t stream);

/* Table width the library picks for a batch of `count` MSMs of n[i] points
 * (host array) over one table. */
int zkp_msm_batch_table_default_window(const uint32_t *n, uint32_t count);

/* Scratch bytes of zkp_msm_batch_table for `count` MSMs of n[i] <= nsrs points
 * (host array) over a table of width window_bits; 0 when they do not fit one
 * pipeline. */
size_t zkp_msm_batch_table_scratch_bytes(const uint32_t *n, uint32_t count, uint32_t nsrs, int window_bits);

/* zkp_msm_batch over a table from zkp_msm_table_build (same nsrs and
 * window_bits): out[i] = sum_{j < n[i]} [scalars[i][j]] bases_j, one bucket set
 * per MSM, one counting sort and accumulation pass for the whole batch. */
cudaError_t zkp_msm_batch_table(void *out, const void *table, uint32_t nsrs, int window_bits, const void *scalars,
                                const uint32_t *n, uint32_t count, void *scratch, size_t scratch_bytes,
                                cudaStream_t stream);

/* Batched NTT of ncols columns (column c at buf + c * col_stride elements)
 * by the natural twiddle table `omegas` (2^log_n entries), optional output
 * scale.  *result_in_tmp (host) tells whether the result is in tmp. */
cudaError_t zkp_ntt_batch(void *buf, void *tmp, const void *omegas, const void *scale, int log_n, uint32_t ncols,
                          size_t col_stride, int *result_in_tmp, cudaStream_t stream);

/* The library's pass split for a transform of 2^log_n points: writes the
 * radices (log2, at most 4) and returns their count (0 if unsupported). */
int zkp_ntt_default_plan(int log_n, int *radices);

/* zkp_ntt_batch with the pass split given (host array of npasses radices,
 * log2, summing to log_n; each in 6..12 when there is more than one pass), for
 * a radix autotuner. */
cudaError_t zkp_ntt_batch_plan(void *buf, void *tmp, const void *omegas, const void *scale, int log_n,
                               uint32_t ncols, size_t col_stride, const int *radices, int npasses,
                               int *result_in_tmp, cudaStream_t stream);

/* out[i] = base * w^i for i < n (base and w device scalars). */
cudaError_t zkp_powers(void *out, const void *base, const void *w, uint32_t n, cudaStream_t stream);

/* Elements of the coset table zkp_extend_batch needs for (log_n, ext_bits). */
size_t zkp_coset_table_elems(int log_n, int ext_bits);

/* Coset-extension tables for the evaluation on shift * <w_N>, w_N a primitive
 * 2^(log_n + ext_bits)-th root of unity (device scalars shift and w_ext), tw the
 * natural w_n table.  With t_j = shift * w_N^j and R = 2^r the second radix of
 * the two-pass plan of 2^log_n: when 2^9 <= R <= 2^11 the table holds
 * W_j[q R + y] = w_n^(q y) t_j^q (2^ext_bits * n entries) followed by
 * S_j[i] = (t_j^(n/R))^i (2^ext_bits * R entries); otherwise it holds the
 * twists t_j^k (2^ext_bits * n entries). */
cudaError_t zkp_coset_twist_tables(void *twist, const void *shift, const void *w_ext, int log_n, int ext_bits,
                                   const void *tw, cudaStream_t stream);

/* Extended-domain phase for ncols columns of 2^log_n Lagrange values:
 *   coeff = iNTT(lagrange)            (tw_inv = natural table of w_n^-1, n_inv)
 *   ext[c][2^e * i + j] = NTT_n(coeff * twist_j)[i]
 * i.e. ext is the evaluation on the coset shift * <w_N>, N = 2^(log_n + e), in
 * natural order.  scratch: ncols * 2^e * n elements.  coeff_out may be NULL
 * only when log_n <= 12 (one pass per transform).  Each stage is one launch
 * over all columns.  stage_events (may be NULL) is an array of 5 cudaEvent_t
 * recorded on `stream` before the first stage, between the stages and after
 * the last, so a caller can time each stage. */
cudaError_t zkp_extend_batch(void *ext_out, void *coeff_out, const void *lagrange_in, uint32_t ncols, int log_n,
                             int ext_bits, const void *tw_inv, const void *n_inv, const void *tw, const void *twist,
                             void *scratch, void *stage_events, cudaStream_t stream);

/* Elements of the table blob of zkp_extend_batch_tables (0 when the sizes are
 * unsupported): every twiddle, twist and scale of the phase as the pair
 * (w, w') with w canonical and w' = floor(w 2^256 / r), two elements an
 * entry: tw at [0, 2n), tw_inv at [2n, 4n), n^-1 at [4n, 4n + 2), then the
 * coset tables of zkp_coset_twist_tables in the same pair layout. */
size_t zkp_extend_table_elems(int log_n, int ext_bits);

/* Fills the blob from the natural tables tw (w_n^i) and tw_inv (w_n^-i), n^-1
 * and the coset generator shift * w_ext^j (all device values in Montgomery
 * form). */
cudaError_t zkp_extend_tables(void *tables, const void *tw, const void *tw_inv, const void *n_inv, const void *shift,
                              const void *w_ext, int log_n, int ext_bits, cudaStream_t stream);

/* zkp_extend_batch over the blob: the same outputs, every product by a table
 * factor computed from the pair (a w - floor(a w' / 2^256) r, 207 instead of
 * 264 integer multiply-adds). */
cudaError_t zkp_extend_batch_tables(void *ext_out, void *coeff_out, const void *lagrange_in, uint32_t ncols,
                                    int log_n, int ext_bits, const void *tables, void *scratch, void *stage_events,
                                    cudaStream_t stream);

/* out[i] = (accumulate ? out[i] : 0) + 1 / (in[i] + c[0]) (c may be NULL);
 * zero maps to zero. out may alias in.  scratch: NULL or
 * zkp_scan_scratch_elems(n) device elements (not aliasing out or in); with it
 * the whole array takes one field inversion instead of one per 2048 elements. */
cudaError_t zkp_batch_inverse(void *out, const void *in, const void *c, uint32_t n, int accumulate, void *scratch,
                              cudaStream_t stream);

/* out[i] = [k64[i]] G as affine points (identity (0, 0) for k = 0), with
 * G = (1, 2) the BN254 G1 generator and k64 a device array of n u64: bases
 * with known discrete logarithms for benchmarks and SRS-style test data. */
cudaError_t zkp_g1_multiples(void *out, const void *k64, uint32_t n, cudaStream_t stream);

/* out[i] = in[i] * R mod r: canonical Fr values (below r) to Montgomery form;
 * out may alias in. */
cudaError_t zkp_fr_to_mont(void *out, const void *in, uint32_t n, cudaStream_t stream);

/* Scratch elements (32 bytes each) the prefix scans need for n elements. */
size_t zkp_scan_scratch_elems(uint32_t n);

/* Exclusive prefix product / sum with carried-in value (init may be NULL):
 * out[i] = init (op) in[0] (op) ... (op) in[i-1]; out may alias in.  Above
 * 2048 elements the product runs in one launch (decoupled look-back over
 * tiles of 2048 elements) and the sum as the sums of 256-element segments,
 * their scan and a scan of each segment from its prefix, one warp a segment
 * (launches that never wait on one another). */
cudaError_t zkp_grand_product(void *out, const void *in, uint32_t n, const void *init, void *scratch,
                              cudaStream_t stream);
cudaError_t zkp_grand_sum(void *out, const void *in, uint32_t n, const void *init, void *scratch,
                          cudaStream_t stream);

/* Waits of the single-pass scans (zkp_grand_product / zkp_grand_sum and the
 * grand products built on them) that ran out of polls since the library was
 * loaded: each took the missing tile as the identity, so a non-zero count
 * means a wrong result.  Synchronous; 0xffffffff if the read failed. */
uint32_t zkp_scan_timeouts(void);

/* Permutation argument, one chunk of ncols columns (src/permutation.rs:16-150):
 * z[0] = *init, z[i+1] = z[i] * prod_c (v_c[i] + dbeta[c]*w^i + gamma) /
 * (v_c[i] + beta*sigma_c[i] + gamma), with dbeta[c] = beta * delta^(offset+c).
 * cols, sigmas: device arrays of ncols device pointers; omegas: w^i table. */
cudaError_t zkp_permutation_z(void *z, const void *cols, const void *sigmas, int ncols, const void *beta,
                              const void *gamma, const void *dbeta, const void *omegas, const void *init, uint32_t n,
                              void *scratch, cudaStream_t stream);

/* Shuffle argument (src/shuffle.rs:143-212): z[0] = 1,
 * z[i+1] = z[i] * prod_g (input_g[i] + betas[g]) / prod_g (table_g[i] + betas[g]).
 * scratch: n + zkp_scan_scratch_elems(n) elements. */
cudaError_t zkp_shuffle_z(void *z, const void *inputs, const void *tables, const void *betas, int groups, uint32_t n,
                          void *scratch, cudaStream_t stream);

/* ----------------------------------------------------------------------
 * Quotient over cosets of the extended domain, and multi-open helpers
 * (csrc/quotient.cu).  They replace the per-column 2^(k+e) extension and the
 * per-family kernels of src/eval_h.rs:410-1199 with per-coset work, and the
 * host-side divisions of src/multiopen.rs:145-159, 543-553.
 * ------------------------------------------------------------------ */

/* NTT of ncols columns from `in` (stride in_stride) into `out` (stride
 * out_stride, out != in): out_c = NTT(in_c[k] * in_mul[k]) (in_mul may be
 * NULL), every output times *scale when scale is non-NULL.  With in_mul[k] =
 * (zeta w_N^j)^k it gives coset j of the extended domain zeta <w_N>
 * (N = E n) from coefficients.  tmp: n * ncols elements (unused for one-pass
 * sizes).  pairs != 0: omegas, in_mul and scale hold (w, w') known-factor
 * pairs (zkp_shoup_pairs), 2 elements an entry. */
cudaError_t zkp_ntt_batch_twisted(void *out, const void *in, void *tmp, const void *omegas, const void *in_mul,
                                  const void *scale, int log_n, uint32_t ncols, size_t in_stride, size_t out_stride,
                                  int pairs, cudaStream_t stream);

/* out[2i], out[2i+1] = (w, w' = floor(w 2^256 / r)) for the Montgomery-form
 * factors in[i], i < n: the table form of products by a known factor. */
cudaError_t zkp_shoup_pairs(void *out, const void *in, uint32_t n, cudaStream_t stream);

/* Arguments of zkp_eval_h_fused.  Every pointer is a device pointer; `T**`
 * fields are device arrays of device pointers.  Row i of every column is row
 * i of one coset (rot_scale 1) or of the whole extended domain (rot_scale E);
 * a rotation r reads row (i + r * rot_scale) mod n. */
typedef struct zkp_eval_h_args {
    uint32_t n;
    int rot_scale;
    const void *y;             /* the challenge y */
    /* gates: [coeff, col, col, ..., NULL, coeff, ...] as field_op_batch_mul_sum
     * takes them, coefficients carrying their powers of y; one rotation per
     * column entry */
    const void *gate_terms;
    const void *gate_rots;
    int gate_terms_n;
    const void *l0, *l_last, *l_active;
    const void *x;             /* the point X of each row (permutation only) */
    const void *beta, *gamma;
    /* permutation: perm_chunks products z_j over chunks of perm_chunk_len of
     * the perm_cols_n columns; perm_dbeta[c] = beta * delta^c (Fr array);
     * perm_last_rot = -(blinding factors + 1) links the chunks */
    int perm_chunks, perm_chunk_len, perm_cols_n, perm_last_rot;
    const void *perm_z, *perm_cols, *perm_sigmas, *perm_dbeta;
    /* logup lookups with one input per set: 4 pointers each, input, table,
     * multiplicity, z */
    int lookups;
    const void *lookup_cols;
    /* shuffles: per shuffle z, then shuffle_group_len[s] (input, table)
     * pairs; shuffle_betas[g] = beta^(g + 1) */
    int shuffles;
    const void *shuffle_cols, *shuffle_group_len, *shuffle_betas;
    const void *scale;         /* optional factor of every output (1 / Z_H on a coset) */
} zkp_eval_h_args;

/* The constraint expression of the prover's quotient over n rows, in one pass
 * that reads each column once and writes h once: the gate terms, then with
 * Horner steps in y the permutation (l_0 (1 - z_0), l_last (z_last^2 -
 * z_last), the chunk links, the chunk products), every logup lookup and every
 * shuffle, exactly the chain that src/eval_h.rs:588-1199 builds with
 * field_op_batch_mul_sum, permutation_eval_h_p1 / p2, field_op, logup_eval_h
 * and shuffle_eval_h_v2 (cuda/bn254.cu:664-1071). */
cudaError_t zkp_eval_h_fused(void *h, const zkp_eval_h_args *args, cudaStream_t stream);

/* From the E = 2^ext_bits coset iNTTs g_j (g_j = iNTT_n of h on coset
 * zeta w_N^j <w_n>, scaled by 1/n; stride g_stride) to the N = E n
 * coefficients of h, with h's values first multiplied by t_j on coset j:
 * out[r + n s] = zeta^-(r+ns) / E * sum_j w_E^-(j s) t_j w_N^-(j r) g_j[r].
 * winv[r] = w_N^-r (n entries); consts = t_0..t_{E-1}, w_E^-k (k < E),
 * zeta^-k / E (k < 3).  ext_bits 1..3.  Equals src/eval_h.rs:463-510
 * (field_mul_zip by t_evaluations, iNTT of 2^(k+e), extended_prepare with
 * to_coset). */
cudaError_t zkp_coset_combine(void *out, const void *g, size_t g_stride, const void *winv, const void *consts,
                              int log_n, int ext_bits, cudaStream_t stream);

/* q = (a(X) - a(z)) / (X - z) for n coefficients: q_i = sum_{j>i} a_j z^(j-i-1),
 * q_{n-1} = 0, the layout src/multiopen.rs:145-159 leaves.  z is a HOST
 * pointer to one Fr (Montgomery form); scratch:
 * zkp_poly_divide_scratch_elems(n) elements; q must not alias a. */
size_t zkp_poly_divide_scratch_elems(uint32_t n);
cudaError_t zkp_poly_divide_linear(void *q, const void *a, const void *z, uint32_t n, void *scratch,
                                   cudaStream_t stream);

/* out[p] = sum_i polys[p][i] * powers[i] for count polynomials of n
 * coefficients (powers: x^i, i < n, from zkp_powers); scratch:
 * zkp_poly_eval_batch_scratch_elems(count) elements. */
size_t zkp_poly_eval_batch_scratch_elems(uint32_t count);
cudaError_t zkp_poly_eval_batch(void *out, const void *polys, uint32_t count, const void *powers, uint32_t n,
                                void *scratch, cudaStream_t stream);

/* No counterpart in the reference.  zkp_msm without caller-supplied scratch,
 * for callers that cannot allocate device memory: a host whose device memory
 * is all owned by its own pool, or a latency-critical path that cannot afford
 * cudaMalloc's implicit device synchronisation.  out (96-byte Jacobian) = sum_i [scalars_i] bases_i for
 * n <= 16384 points; larger n returns cudaErrorInvalidValue without launching.
 * The scratch is a 9 MiB __device__ array inside the library (one per GPU
 * that loads it, held until exit) shared by every call: calls that overlap on
 * the GPU race, so order them on one stream.  The first call on a device looks
 * up the array's address (cudaGetSymbolAddress) and should come before any
 * stream capture.  It calls no allocating routine: no cudaMalloc, no
 * cudaFree, no cudaMallocAsync. */
cudaError_t zkp_msm_static(void *out, const void *bases, const void *scalars, uint32_t n, cudaStream_t stream);

/* ----------------------------------------------------------------------
 * MSM schedule selection (no counterpart in the reference, whose window width
 * is the fixed formula of src/cuda/msm.rs:105).  The schedule only picks the
 * window width; results never depend on it.
 * -------------------------------------------------------------------- */

/* Bit-length histogram of n Montgomery-form scalars, accumulated into
 * hist[0..6] (device u32): zero, 1-16, 17-32, 33-64, 65-128, 129-192, 193-254. */
cudaError_t zkp_scalar_histogram(const void *scalars, uint32_t n, uint32_t *hist, cudaStream_t stream);

/* Exhaustive search: times zkp_msm for each window c in [c_min, c_max] whose
 * scratch fits, reps runs after one warm-up, times_ms[c - c_min] = mean ms or
 * -1 when skipped; returns the fastest c (-1 on error).  out: 96-byte result.
 * Synchronises the stream. */
int zkp_msm_autotune(const void *bases, const void *scalars, uint32_t n, int c_min, int c_max, int reps,
                     void *scratch, size_t scratch_bytes, float *times_ms, void *out, cudaStream_t stream);

/* MLP cost model (FP32, inputs -> 64 -> 64 -> 1, ReLU) predicting log(ms) of
 * one MSM from [log2 n / 24, log2 batch / 8, 7 histogram fractions,
 * (c - 12) / 8].  Parameters, gradients and Adam moments are device float
 * arrays of zkp_mlp_param_count() entries; X is B x zkp_mlp_input_dim(). */
int zkp_mlp_input_dim(void);
size_t zkp_mlp_param_count(void);
size_t zkp_mlp_scratch_floats(uint32_t B);
cudaError_t zkp_mlp_init(float *params, uint64_t seed, cudaStream_t stream);
cudaError_t zkp_mlp_forward(const float *params, const float *X, uint32_t B, float *y, cudaStream_t stream);
/* mean squared error over the batch, each sample's squared error scaled by
 * weights[b] (device floats; null = all 1), and its gradient (loss: device
 * float) */
cudaError_t zkp_mlp_grad(const float *params, const float *X, const float *t, const float *weights, uint32_t B,
                         float *grads, float *loss, float *scratch, cudaStream_t stream);
/* one Adam step, step >= 1 */
cudaError_t zkp_mlp_train_step(float *params, float *grads, float *m, float *v, const float *X, const float *t,
                               const float *weights, uint32_t B, float lr, int step, float *loss, float *scratch,
                               cudaStream_t stream);
/* window with the smallest predicted time for the nine shape features
 * (host array); scratch: 256 device floats; synchronises the stream */
int zkp_msm_schedule_predict(const float *params, const float *features, int c_min, int c_max, float *scratch,
                             cudaStream_t stream);

/* ======================================================================
 * Part 3: calibration
 * ==================================================================== */

/* Runs blocks x 256 threads, each 4 independent chains of `iters` dependent
 * Fr Montgomery products (4 * iters * blocks * 256 products in total); timed
 * by the caller, this is the integer-pipe roofline denominator for the NTT
 * and MSM kernels.  `out` (one element) is written only if the result is 0. */
cudaError_t zkp_calib_mont_rate(void *out, uint32_t blocks, uint32_t iters, cudaStream_t stream);

/* The same for products by a known factor (the (w, w') pair at `pair`, the
 * product form of zkp_extend_batch_tables). */
cudaError_t zkp_calib_shoup_rate(void *out, const void *pair, uint32_t blocks, uint32_t iters, cudaStream_t stream);

/* ======================================================================
 * Part 4: host staging (replaces src/hugetlb.rs and src/async_copy_queue.rs)
 * ==================================================================== */

/* Host memory pool handing out chunks of chunk_bytes (rounded up to 4 KiB)
 * from blocks of chunks_per_block chunks.  flags: 1 = page-lock each block
 * with cudaHostRegister (what src/hugetlb.rs registers), 2 = map blocks with
 * huge pages (MAP_HUGETLB, else transparent huge pages are requested).
 * Thread-safe; NULL on failure. */
void *zkp_host_pool_create(size_t chunk_bytes, int chunks_per_block, int flags);
/* one chunk (bytes <= chunk_bytes) or NULL */
void *zkp_host_pool_alloc(void *pool, size_t bytes);
/* 0, or -1 for a pointer the pool did not hand out (or freed twice) */
int zkp_host_pool_free(void *pool, void *ptr);
/* blocks mapped so far and chunks handed out (either pointer may be NULL) */
void zkp_host_pool_stats(void *pool, size_t *blocks, size_t *used_chunks);
void zkp_host_pool_destroy(void *pool);

/* Bounded asynchronous copy queue on `device` (src/async_copy_queue.rs): at
 * most max_in_flight copies in flight, each on its own stream.  NULL on
 * failure.  The caller's current device is unchanged on return.  One owner
 * thread. */
void *zkp_copy_queue_create(int max_in_flight, int device);
/* one cudaMemcpyAsync of `bytes` (kind: a cudaMemcpyKind value), ordered
 * after the work already queued on `after`; when max_in_flight copies are in
 * flight, first waits for the oldest.  Host buffers should come from a
 * page-locked pool for the copy to be asynchronous. */
cudaError_t zkp_copy_queue_push(void *queue, void *dst, const void *src, size_t bytes, int kind,
                                cudaStream_t after);
/* waits for every copy in flight */
cudaError_t zkp_copy_queue_sync(void *queue);
void zkp_copy_queue_destroy(void *queue);

#ifdef __cplusplus
}
#endif

#endif
