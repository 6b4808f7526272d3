/* nrgb.h - C ABI of the B200 NRG step library (libnrgb.so).
 *
 * Plain pointers and sizes only.  All matrices are column-major FP64.
 * Every function returns 0 on success or a nonzero status; the message of the
 * last failure on a context is available from nrgb_last_error().  The
 * library never calls exit(); a caller that wants the reference's behaviour
 * on LAPACK failure (src/portabil.h:130-140 my_error -> exit(1)) maps a
 * nonzero status to its own error path.
 *
 * Seams of the reference that these entry points replace:
 *   nrgb_syev_batched      dsyev_('V','L',...) per invariant subspace
 *                          (src/diag.h:9-10, 54-89; called per block from
 *                          src/nrg.cc:2484-2507), here for a whole step at once.
 *   nrgb_gemm_grouped_dev  atlas::gemm / cblas dgemm calls of the operator
 *                          recalculation and density-matrix updates
 *                          (src/recalc.cc:90-91, 268-272; src/dmnrg.h:382-387).
 *   nrgb_run               the `nrg` executable's main program for the NRG
 *                          iteration (src/nrg.cc:3429-3469 start_calculation):
 *                          reads `param` and `data`, writes `td`, spectra.
 */
#ifndef NRGB_H
#define NRGB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nrgb_ctx nrgb_ctx;

/* Context bound to one CUDA device; owns all device memory it allocates. */
int nrgb_create(int device, nrgb_ctx** out);
int nrgb_destroy(nrgb_ctx* ctx);
const char* nrgb_last_error(const nrgb_ctx* ctx);
const char* nrgb_version(void);

/* Eigen-decomposition of a batch of dense symmetric blocks (host memory).
 * a[b]: n[b] x n[b] column-major, both triangles filled; on return it holds the
 *       eigenvectors (column r belongs to w[b][r]), as dsyev('V') does.
 * w[b]: n[b] eigenvalues in ascending order.
 * Replaces one dsyev_ call per block (src/diag.h:54-89). */
int nrgb_syev_batched(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a,
                      double* const* w);

/* Same on device memory: a_dev[b] is destroyed, z_dev[b] (n x n, must not alias
 * a_dev[b]) receives the eigenvectors, w_dev[b] the eigenvalues.  Runs on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and returns after
 * the work completed. */
int nrgb_syev_batched_dev(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a_dev,
                          double* const* w_dev, double* const* z_dev, void* stream);

/* One product term of a grouped GEMM:  alpha * op(A) * op(B),
 * op(A) m x k, op(B) k x n, trans = 0 (as stored) or 1 (transposed). */
typedef struct {
  const double* a;
  const double* b;
  int lda, ldb, k, trans_a, trans_b;
  double alpha;
} nrgb_gemm_term;

/* Output of a grouped GEMM:  C = beta*C + sum of terms[term0 .. term0+nterms). */
typedef struct {
  double* c;
  int ldc, m, n;
  double beta;
  int term0, nterms;
} nrgb_gemm_out;

/* Grouped FP64 GEMM on device pointers (descriptors in host memory). */
int nrgb_gemm_grouped_dev(nrgb_ctx* ctx, int nout, const nrgb_gemm_out* outs, int nterms,
                          const nrgb_gemm_term* terms, void* stream);

/* ---- Step-level plan: the reference's own driver and Symmetry plug-ins
 * call the device one NRG step at a time.  nrg_iterate (src/nrg.cc:3043-3051)
 * and the Symmetry class (src/symmetry.cc:64-221, sym-<SYM>.cc,
 * nrg-recalc-<SYM>.cc) stay on the host; they expand their tables into the
 * flat task lists below, so a new symmetry needs host tables only.  Energies,
 * eigenvectors and operator blocks stay in device memory under integer
 * handles owned by the context. */

/* Device matrices (column-major).  nrgb_mat_upload copies rows x cols
 * doubles from host memory; nrgb_mat_download copies back; nrgb_run_begin
 * frees every handle of the context and resets the splitting-correction map
 * (the reference keeps it for a whole run, src/splitting.cc). */
int nrgb_mat_upload(nrgb_ctx* ctx, int rows, int cols, const double* host, int* handle);
int nrgb_mat_download(nrgb_ctx* ctx, int handle, double* host);
int nrgb_mat_shape(nrgb_ctx* ctx, int handle, int* rows, int* cols);
int nrgb_mat_free(nrgb_ctx* ctx, int handle);
int nrgb_run_begin(nrgb_ctx* ctx);

/* Diagonal term of block blk (diag_function, src/matrix.cc:172-192 and the
 * sqrt(Lambda) E_prev diagonal of src/nrg.cc:2456-2478):
 *   H[off + r, off + r] += scale * src[r] + shift,  r < len
 * (src: handle of a vector of at least len values, or -1 for shift only). */
typedef struct {
  int blk, off, len, src;
  double scale, shift;
} nrgb_diag_term;
/* Off-diagonal term (offdiag_build, src/matrix.cc:86-137):
 *   H[offi + r, offj + c] += factor * src(r, c)  and the mirror entry,
 * src: handle of a rows x cols matrix (an <I||f||J> block), or -1 for the
 * identity of a square sub-block (diag_offdiag_function,
 * src/matrix.cc:256-276: SPSU2's on-site pairing).  Terms add: a sub-block
 * may take several (SPSU2's hopping and anomalous hopping); the row range
 * [offi, offi+rows) and the column range [offj, offj+cols) must not overlap,
 * and two terms of one block cover the same sub-block or disjoint ones. */
typedef struct {
  int blk, offi, offj, rows, cols, src;
  double factor;
} nrgb_offdiag_term;
typedef struct {
  int nblocks;
  const int* dim;  /* block dimensions */
  int ndiag;
  const nrgb_diag_term* diag;
  int noff;
  const nrgb_offdiag_term* off;
  /* truncation (src/nrg.cc:1919-1998, src/splitting.cc) */
  double fixeps, keepenergy;
  int keep, keepmin;
  double safeguard;
  int safeguardmax;
  int keep_all; /* keep every state (the last step of a CFS/FDM run) */
  double betabar;
} nrgb_step_plan;
/* One NRG step on the device: assemble every block, diagonalise all of them
 * (dsyev per block, src/diag.h:54-89), subtract the ground-state energy,
 * apply the splitting correction and choose the retained states.  Outputs
 * per block b: z_handles[b] (dim x dim eigenvectors, eigenvector r in column
 * r), w_handles[b] (dim eigenvalues, ascending, ground state subtracted,
 * corrected), kept[b]; egs (the subtracted ground-state energy) and, if not
 * NULL, zsums[3b .. 3b+2] = sum_r e^(-betabar E_r), sum_r betabar E_r
 * e^(-betabar E_r), sum_r (betabar E_r)^2 e^(-betabar E_r) over all states of
 * block b (nrg_calculate_TD, src/nrg.cc:2333-2369). */
int nrgb_step(nrgb_ctx* ctx, const nrgb_step_plan* plan, int* z_handles, int* w_handles, int* kept,
              double* egs, double* zsums);

/* Recalculation (recalc_general / recalc_f, src/recalc.cc:12-97, 164-281):
 * output o (k1 x kp) = sum over its terms of
 *   factor * Z1[off1 : off1+r1, 0 : k1]^T * op[0 : r1, 0 : rp] * Zp[offp : offp+rp, 0 : kp]
 * with op = -1 meaning the identity (recalc_f, r1 == rp).  Z1, Zp: the
 * eigenvector handles of nrgb_step (the reference's U blocks of
 * split_in_blocks are these sub-blocks, transposed).  out_handles[o]
 * receives a new handle per output. */
typedef struct {
  int z1, off1, r1;
  int zp, offp, rp;
  int op;
  double factor;
} nrgb_recalc_term;
typedef struct {
  int k1, kp;
  int term0, nterms;
} nrgb_recalc_out;
int nrgb_recalc(nrgb_ctx* ctx, int nout, const nrgb_recalc_out* outs, int nterms, const nrgb_recalc_term* terms,
                int* out_handles);

/* Density-matrix backward step (calc_densitymatrix, src/dmnrg.h:327-475; the
 * DM-NRG and FDM sweeps of src/nrg.cc:1877-1913):
 * output o (r1 x rp) = sum over its terms of
 *   factor * Z1[off1 : off1+r1, 0 : k1] * rho[0 : k1, 0 : kp] * Zp[offp : offp+rp, 0 : kp]^T
 * the adjoint of nrgb_recalc's product: the eigenvector sub-blocks of the
 * subspaces of step N+1 carry their density matrices rho (k1 x kp kept
 * states) back to the sub-blocks of their ancestors at step N.  Z1, Zp:
 * eigenvector handles of nrgb_step; rho: any matrix handle.  out_handles[o]
 * receives a new handle per output. */
typedef struct {
  int z1, off1, k1;
  int zp, offp, kp;
  int rho;
  double factor;
} nrgb_dm_term;
typedef struct {
  int r1, rp;
  int term0, nterms;
} nrgb_dm_out;
int nrgb_dm_backward(nrgb_ctx* ctx, int nout, const nrgb_dm_out* outs, int nterms, const nrgb_dm_term* terms,
                     int* out_handles);

/* FDM spectral weights of one step (SPEC_FDMgt + SPEC_FDMls,
 * src/spec_FDM.cc:41-119) for a list of block pairs (ket block i, bra block
 * j): the greater and lesser sums over the discarded and kept sectors, at
 * the energies E_j - E_i, binned on the logarithmic grid of
 * src/bins.h:22-131 (lowest point 10^floor(log10 emin), bins_per_decade,
 * highest 10^ceil(log10 emax); nbins must equal
 * (int)((ceil(log10 emax) - floor(log10 emin)) * bins_per_decade + 1)) and
 * ADDED to bins[0 .. 2*nbins) (host memory: positive energies, then
 * negative ones, each nbins long).  Weights below discard * |E| are dropped
 * (discard_immediately).  op1, op2: the blocks <j|O1|i>, <j|O2|i>
 * (allj x alli); rho_i, rho_j: the density matrices of the kept states
 * (reti x reti, retj x retj; unused when reti / retj is 0, as at the last
 * step); e_i, e_j: the absolute energies of both blocks' states (shifted by
 * the ground state of the whole run), alli and allj values; factor: the
 * symmetry's spectral-density factor.  T: temperature; wn: the step's
 * weight w_N (src/dmnrg.h:487-596); fermionic: 1 for fermionic operators
 * (the lesser sum enters with +), 0 for bosonic. */
typedef struct {
  int op1, op2;
  int rho_i, rho_j;
  int e_i, e_j;
  int reti, retj;
  double factor;
} nrgb_fdm_pair;
int nrgb_spectrum_fdm(nrgb_ctx* ctx, int npairs, const nrgb_fdm_pair* pairs, double T, double wn, int fermionic,
                      double bins_per_decade, double emin, double emax, double discard, int nbins, double* bins);

/* DM-NRG spectral weights of one step (SPEC_DMNRG::calc,
 * src/spec_DMNRG.cc:13-52) for a list of block pairs (ket block p, bra block
 * 1) over their kept states: w = factor * (op1 (op2 rho_p) + s op2 (rho_1
 * op1)) elementwise, s = +1 for fermionic operators and -1 for bosonic, at
 * E = E_1 - E_p, kept where ewin_min <= |E| <= ewin_max (the step's window,
 * src/spectrumrealfreq.cc) and binned at scale * E on the grid of
 * nrgb_spectrum_fdm, ADDED to bins.  rho_1, rho_p: the density matrices of
 * the kept states (dim1 x dim1, dimp x dimp; their sizes give the kept
 * counts); op1, op2: the blocks <1|O|p> (at least dim1 x dimp, same shape);
 * e_1, e_p: the step's energies (at least dim1 / dimp values). */
typedef struct {
  int op1, op2;
  int rho_1, rho_p;
  int e_1, e_p;
  double factor;
} nrgb_dmnrg_pair;
int nrgb_spectrum_dmnrg(nrgb_ctx* ctx, int npairs, const nrgb_dmnrg_pair* pairs, double scale, double ewin_min,
                        double ewin_max, int fermionic, double bins_per_decade, double emin, double emax,
                        double discard, int nbins, double* bins);

/* Split-precision form of nrgb_gemm_grouped_dev (same descriptors): every
 * product is computed from `slices` (2..8) signed 7-bit slices of each
 * operand, with power-of-two scales per row of op(A) and per column of op(B),
 * as exact INT8 tensor-core products (tcgen05 kind::i8, INT32 accumulators)
 * recombined in FP64 with a compensated sum.  The error of an entry is about
 * k * 2^-7S * (S + 3) * max|op(A) row| * max|op(B) column|; S = 8 is at the
 * level of an FP64 product.  Replaces the BLAS gemm of the recalculation
 * (src/recalc.cc:268-272) and the density matrices (src/dmnrg.h:382-387) in
 * the split-precision form.  Returns after the work completed. */
int nrgb_gemm_grouped_split_dev(nrgb_ctx* ctx, int slices, int nout, const nrgb_gemm_out* outs, int nterms,
                                const nrgb_gemm_term* terms, void* stream);

/* The two hot operations of one NRG step on a batch of blocks, host memory:
 * eigen-decomposition of every block h[b] (n[b] x n[b], column-major,
 * symmetric; not modified) into w[b] (ascending) and eigenvectors Z_b, then
 * for every operator o the basis change
 *     out[o] = Z_{bra[o]}^T * op[o] * Z_{ket[o]}     (n[bra] x n[ket]),
 * which is the per-table-row contraction U1 * O * Up^T of the reference's
 * recalc_general (src/recalc.cc:268-272) after dsyev (src/diag.h:54-89).
 * z[b] may be NULL (eigenvectors not returned). */
int nrgb_eig_recalc_step(nrgb_ctx* ctx, int nblocks, const int* n, const double* const* h,
                         double* const* w, double* const* z, int nops, const int* bra, const int* ket,
                         const double* const* op, double* const* out);

/* Same with device pointers; a_dev[b] holds the block on entry and is
 * destroyed, z_dev[b] receives the eigenvectors.  Runs on `stream`. */
int nrgb_eig_recalc_step_dev(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a_dev,
                             double* const* w_dev, double* const* z_dev, int nops, const int* bra,
                             const int* ket, const double* const* op_dev, double* const* out_dev,
                             void* stream);

/* Launch accounting: enable != 0 turns on per-kernel timing with CUDA events
 * (and resets all counters); enable == 0 turns it off. */
int nrgb_profile(nrgb_ctx* ctx, int enable);
/* As nrgb_profile(ctx, 1), but only launches of kernel `name` (or of a prefix
 * ending in '*') are timed; all launches are still counted.  Each timed
 * launch records two CUDA events, so timing every launch of a many-threaded
 * caller (a run server) slows it down; timing one kernel keeps that cost to
 * its own launches.  No counterpart in the reference. */
int nrgb_profile_only(nrgb_ctx* ctx, const char* name);
/* Launches and total device milliseconds of kernel `name` since the last
 * nrgb_profile call ("*" = all kernels of the library; ms is 0 unless timing
 * is on).  Names: trd_panel, gemm_f64, syev_small, dc_*, bt_*, assemble_*,
 * spec_dmnrg, spec_fdm, merge_bins, gather_diag, col_scale. */
int nrgb_kernel_stats(nrgb_ctx* ctx, const char* name, long* launches, double* ms);
/* Algorithmic work stated by the host code for the launches counted under
 * `name` (same name matching): bytes for trd_panel (each column's trailing
 * block read once), flops (2 m n k) for the gemm_f64* call sites.  Counted
 * since the last nrgb_profile(ctx, 1). */
int nrgb_kernel_work(nrgb_ctx* ctx, const char* name, double* units);

/* Allocation-free basis change, device pointers:
 *     out[o] = Z_bra[o]^T * op[o] * Z_ket[o]
 * (Z_bra[o]: n_bra[o] x n_bra[o], op[o]: n_bra[o] x n_ket[o],
 *  Z_ket[o]: n_ket[o] x n_ket[o], out[o]: n_bra[o] x n_ket[o], column-major).
 * This entry point has no counterpart in the reference.  It is for callers
 * that must not see the library allocate device memory: a host that owns the
 * device-memory budget (e.g. a serving loop that admits runs by projected
 * footprint) or a loop that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree.  It needs no context and calls no allocator: its
 * intermediates and launch descriptors live in a fixed 32 MiB device array
 * inside the library, which every GPU that loads the library holds until the
 * process exits.  Limits: at most 1024 operators, and the descriptors plus all
 * n_bra*n_ket intermediates (each rounded up to 256 bytes) must fit in 32 MiB.
 * The first call on a device looks up the array's device address (set-up);
 * make that first call before any stream capture.  Calls share the array, so
 * one call runs at a time per process: a process-wide lock serialises the
 * calls and each call blocks until its work on `stream` has finished (the
 * call is synchronous, whatever stream it is given).  A call on a stream that
 * is capturing returns 7 and enqueues nothing, leaving the capture intact.
 * Returns 0 on success, 1 for invalid arguments, 5 when the sizes exceed the
 * limits above, 6 on a CUDA error, 7 when `stream` is capturing. */
int nrgb_basis_change_noalloc(int nops, const int* n_bra, const int* n_ket, const double* const* z_bra,
                              const double* const* z_ket, const double* const* op, double* const* out,
                              void* stream);

/* Full NRG run of the QS symmetry on the GPU: reads workdir/param and
 * workdir/data, writes td, custom, annotated.dat (if requested) and the
 * spectral-function files into outdir.  stats (may be NULL) receives
 * [0] wall seconds, [1] eigensolver seconds, [2] recalc seconds,
 * [3] density-matrix seconds, [4] spectral seconds, [5] kernels launched,
 * [6] host->device bytes, [7] device->host bytes. */
int nrgb_run(nrgb_ctx* ctx, const char* workdir, const char* outdir, double* stats);

/* Size-bucketed schedule of the batched step, one table per device shared
 * by every context of the process (no counterpart in the reference, whose
 * only schedule is a sort of the blocks by size, src/nrg.cc:2785-2803):
 *   cluster_limit    blocks up to this size are tridiagonalised whole in one
 *                    thread-block cluster, larger ones take cooperative
 *                    panel launches until their trailing block is this small
 *                    (0 = the cluster kernel's capacity);
 *   gemm_large_from  grouped FP64 GEMM launches whose problems average at
 *                    least this output edge use 128 x 128 tiles (0 = never).
 * nrgb_autotune measures both choices on the device (a few seconds of
 * synthetic work: square GEMMs of edge 128..2048 with both tile sizes, one
 * batched eigensolve of a mix of block sizes under several limits), sets the
 * table and writes a JSON report of the timings and choices into `report`
 * (report_len bytes, NUL-terminated, may be NULL).  nrgb_set_schedule sets
 * the table directly (e.g. to replay a tuned schedule); nrgb_get_schedule
 * reads it and the cluster kernel's capacity. */
int nrgb_autotune(nrgb_ctx* ctx, char* report, int report_len);
int nrgb_set_schedule(nrgb_ctx* ctx, int cluster_limit, int gemm_large_from);
int nrgb_get_schedule(nrgb_ctx* ctx, int* cluster_limit, int* gemm_large_from, int* cluster_capacity);

/* Failure detection of the device waits.  Every wait of a kernel in this
 * library is bounded: a grid-barrier wait of the cooperative tridiagonalisation
 * gives up after 2^poll_log2 polls (default 23, about a second), the launch
 * ends early, and the call returns status 2 with "grid barrier timed out"
 * while the context stays usable.  poll_log2 in [4, 30].  No counterpart in
 * the reference (its LAPACK calls have no waits to bound). */
int nrgb_set_wait_limit(nrgb_ctx* ctx, int poll_log2);
/* Host-side fault injection for tests of that path: while `on`, the panel
 * launches' barriers expect one CTA more than is launched (a CTA that never
 * arrives), so their waits run out and nrgb_syev_batched / nrgb_run return
 * the timeout error.  No counterpart in the reference. */
int nrgb_inject_barrier_shortfall(nrgb_ctx* ctx, int on);

/* Eigensolver structure of nrgb_run and nrgb_eig_recalc_step(_dev) on this
 * context: 0 (default) solves all blocks of a step in one batched call; 1
 * makes one solver call per block,
 * the structure of the reference's per-subspace dsyev loop
 * (src/nrg.cc:2484-2507), for comparisons.  Results agree to rounding. */
int nrgb_set_eig_mode(nrgb_ctx* ctx, int mode);

/* ---------------------------------------------------------------------------
 * Run server: many NRG runs in flight on one GPU (continuous batching).
 * No counterpart in the reference, which runs one calculation per process
 * (src/nrg.cc:3429-3469); each run is what nrgb_run does for one work
 * directory, with the same outputs.
 *
 * Requests queue in submission order.  A worker slot (max_runs of them)
 * admits the head of the queue when its projected device bytes
 * (nrgb_project_bytes) fit in mem_budget_bytes beside the runs already
 * admitted; a run is always admitted when no other runs.  Admitted runs
 * execute concurrently, each on its own stream; the block eigensolves of
 * all runs in their first sweep are merged into shared batched solver
 * calls, which wait at most batch_window_us for every such run to queue its
 * blocks.  All calls are thread-safe.
 * ------------------------------------------------------------------------- */
typedef struct nrgb_server nrgb_server;

/* Admission projection, never above the upper bound nrgb_project_bytes:
 * twice the largest measured peak / bound ratio of finished runs of the same
 * shape (keep, chain length, channels, operators, density-matrix kind)
 * times the bound; four times the largest ratio of any shape while none of
 * this shape has finished; the bound while no run has finished.  A run that
 * runs out of device memory on a learned projection is queued once more,
 * first, on the bound.
 * mem_budget_bytes <= 0: 85% of the device memory free at creation.
 * Returns 0, 1 (bad arguments), 2 (CUDA error), 3 (no device), 4 (bad device). */
int nrgb_server_create(int device, int max_runs, double mem_budget_bytes, double batch_window_us,
                       nrgb_server** out);
/* Queue a run; *ticket (>= 1) identifies it.  Returns 0, 1, or 2 when the
 * input cannot be read (text via nrgb_server_error(srv, 0)). */
int nrgb_server_submit(nrgb_server* srv, const char* workdir, const char* outdir, long long* ticket);
/* Wait for a run (timeout_s < 0: no limit).  Returns 0 (done), 2 (the run
 * failed; text via nrgb_server_error(srv, ticket)), 7 (timed out), 1 (unknown
 * ticket).  stats (may be NULL) receives 14 values: the 8 of nrgb_run, then
 * [8] latency from submission to completion (s), [9] queue wait from
 * submission to admission (s), [10] projected bytes, [11] peak device bytes
 * the run's data held, [12] eigensolver calls, [13] admission order. */
int nrgb_server_wait(nrgb_server* srv, long long ticket, double timeout_s, double* stats);
/* Error text of a failed ticket, or of the last failed call when ticket <= 0;
 * valid until the server is destroyed. */
const char* nrgb_server_error(nrgb_server* srv, long long ticket);
/* out[8]: runs done, runs failed, merged eigensolver calls, eigensolver
 * requests, blocks solved, most runs in flight at once, most projected bytes
 * admitted at once, memory budget. */
int nrgb_server_counters(nrgb_server* srv, double* out);
/* Finishes every queued and running request, then frees the server. */
int nrgb_server_destroy(nrgb_server* srv);
/* Upper bound of the device bytes a run of workdir holds at once, from
 * workdir/param and workdir/data (host only; no device needed).
 * Returns 0, 1 (bad arguments) or 2 (input not readable). */
int nrgb_project_bytes(const char* workdir, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* NRGB_H */
