/*
 * gb200.h — C ABI of the B200 density-fitted GW / HF / Dyson engine.
 *
 * Plain C: opaque context, plain pointers and sizes, int status codes.  Complex
 * numbers are interleaved (re, im) pairs of double, arrays are row-major with
 * the reference's index order.  Every "host" entry point takes host pointers,
 * copies to the GPU, computes and copies back; every "_device" entry point
 * takes device pointers and a cudaStream_t passed as void*.
 *
 * The entry points replace the reference's kernel plug-in interface
 * (green-mbpt, src/green/mbpt/kernel_factory.h:28-36,44-108):
 *   custom_gw_kernel -> callback (G, Sigma)  ==> gb200_gw_sigma
 *   custom_hf_kernel -> callback (dm) -> F    ==> gb200_hf_fock
 * and the Dyson step of src/dyson.cpp (find_mu :101-174, compute_G :176-288)
 * plus compute_energy of src/common_utils.cpp:5-55.
 */
#ifndef GB200_H
#define GB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The C++ plug-in shim maps them onto the reference's
 * exception classes (src/green/mbpt/except.h:28-56). */
#define GB200_OK 0
#define GB200_ERR_INVALID 1          /* bad argument or shape -> mbpt_kernel_error */
#define GB200_ERR_WRONG_GRID 2       /* odd number of tau points -> mbpt_wrong_grid */
#define GB200_ERR_MU_SEARCH 3        /* stalled bisection -> mbpt_chemical_potential_search_failure */
#define GB200_ERR_OUTDATED_INPUT 4   /* integral format version too old -> mbpt_outdated_input */
#define GB200_ERR_CUDA 5             /* CUDA runtime / launch failure -> mbpt_kernel_error */
#define GB200_ERR_OOM 6              /* device allocation failed -> mbpt_kernel_error */
#define GB200_ERR_STATE 7            /* required set-up call missing -> mbpt_kernel_error */
#define GB200_ERR_NONFINITE 8        /* NaN/Inf found in a result -> mbpt_kernel_error */

/* Contraction precision for the P0 and Sigma contractions. */
#define GB200_PREC_FP64 0            /* plain FP64 (the oracle-parity path) */
#define GB200_PREC_SPLIT 1           /* Ozaki-sliced INT8 tensor-core products, FP64 recombination */

/* Which DF integral set a call refers to (dfintegral_file vs dfintegral_hf_file, common_defs.h:156-157). */
#define GB200_INTEGRALS_GW 0
#define GB200_INTEGRALS_HF 1

typedef struct gb200_context gb200_context;

/* Problem dimensions (the constructor arguments of gw_cpu_kernel / hf_kernel,
 * src/green/mbpt/kernels.h:42-53,186-189).  No point-group symmetry: every
 * k-point is irreducible (ink = nk). */
typedef struct {
  int32_t nk;      /* k-points of the full mesh */
  int32_t nao;     /* atomic orbitals */
  int32_t nso;     /* spin orbitals: nao, or 2 nao with ns = 1 for two-component (X2C) input
                      (spinor blocks aa, ab, ba, bb of nao x nao; integrals stay nao x nao) */
  int32_t ns;      /* spin channels, 1 or 2 */
  int32_t NQ;      /* auxiliary basis size */
  int32_t nts;     /* tau points (even) */
  int32_t nw;      /* fermionic Matsubara samples */
  int32_t nw_b;    /* bosonic Matsubara samples */
  double beta;     /* inverse temperature */
} gb200_dims;

/* Library version string and the integral-format version it accepts
 * (INPUT_VERSION, common_defs.h:35; CheckVersion :191-212). */
const char* gb200_version(void);
int gb200_check_integral_version(const char* version);

/* Create / destroy a context bound to CUDA device `device`.
 * Replaces the kernel object built by gw_kernel_factory::get_kernel /
 * hf_kernel_factory::get_kernel (kernel_factory.h:44-108). */
int gb200_create(const gb200_dims* dims, int device, gb200_context** out);
void gb200_destroy(gb200_context* ctx);
const char* gb200_last_error(const gb200_context* ctx);

/* k/q maps of brillouin_zone_utils::k_q_map (call sites gw_cpu_kernel.cpp:90,117):
 * kplus[k*nk+q] = k1_from_k2q(k, q), kminus[k*nk+q] = k2_from_k1q(k, q). */
int gb200_set_kq_maps(gb200_context* ctx, const int32_t* kplus, const int32_t* kminus);

/* Imaginary-time transforms of transformer_t as dense complex matrices:
 * Tnt_f [nw,nts], Ttn_f [nts,nw], Tnt_b [nw_b,nts], Ttn_b [nts,nw_b];
 * wsample_f [nw] fermionic frequencies (real omega_n). */
int gb200_set_grid(gb200_context* ctx, const double* Tnt_f, const double* Ttn_f, const double* Tnt_b,
                   const double* Ttn_b, const double* wsample_f);

/* DF integrals V^Q_ij(k1,k2) in the reference's stored form: only k1 >= k2 at
 * pair index k1*(k1+1)/2 + k2, shape [nk(nk+1)/2, NQ, nao, nao]
 * (df_integral_t.h:64-92,162-177).  `which` = GB200_INTEGRALS_GW / _HF. */
int gb200_set_integrals(gb200_context* ctx, int which, const double* V_half, int64_t npairs);

/* The same integrals from device memory, in chunks: V_dev holds the stored pairs
 * [pair_begin, pair_begin + pair_count) of the layout above.  A call with
 * pair_begin = 0 starts a new set; the set is usable once every stored pair has
 * been delivered.  `stream` is a cudaStream_t (or NULL for the context's stream). */
int gb200_set_integrals_device(gb200_context* ctx, int which, const double* V_dev, int64_t pair_begin,
                               int64_t pair_count, void* stream);

/* Restrict the q loop to [q_begin, q_end): one shard of the reference's internode q
 * distribution (gw_cpu_kernel.cpp:45-48).  Sigma then holds this shard's partial sum,
 * already divided by nk, and the shards of all ranks add up to the full self-energy
 * (the allreduce of :53-54).  Default: all q. */
int gb200_set_q_range(gb200_context* ctx, int q_begin, int q_end);

/* The self-energies of n contexts (independent systems of any shapes, one device) in one call:
 * G_dev[i] and Sigma_dev[i] are device buffers of context i, as for gb200_gw_sigma_device.  The
 * systems' q-points run in step (round r takes the r-th q-point of every system that has one, the
 * k-blocks in step), and each contraction stage of a round is one grouped persistent tensor-core
 * launch over the tiles of all systems when all of them use split precision with the same slice
 * count.  Every system's result is the one gb200_gw_sigma_device gives it alone.  Errors are
 * reported on ctxs[0]. */
int gb200_gw_sigma_batch_device(gb200_context* const* ctxs, int n, const double* const* G_dev,
                                double* const* Sigma_dev, void* stream);

/* Column tile width of the split-precision contractions of a context (a multiple of 16, at most
 * the widest tile that S slices allow; 0: the widest).  The batched workload's autotuner picks it
 * per (nao, naux). */
int gb200_set_tile_width(gb200_context* ctx, int bn);

/* q-sharded storage of the GW integrals: only the stored pairs `pair_ids` (indices
 * k1*(k1+1)/2 + k2 with k1 >= k2, strictly increasing; `count` of them) with their blocks
 * V_pairs [count, NQ, nao, nao] in that order, host memory (on_device = 0) or device memory
 * (on_device = 1, `stream` as for gb200_set_integrals_device).  A rank whose q range is
 * [q_begin, q_end) needs the pairs {k, k+q} of those q for every k: the reference's node split
 * reads exactly the k-pairs of its q-points (gw_cpu_kernel.cpp:45-48,88-90,113-119 through
 * df_integral_t::read_integrals, df_integral_t.h:64-84).  The context then holds 2 count - (diagonal
 * pairs) blocks instead of nk^2.  gw_sigma and hf_fock refuse (GB200_ERR_STATE) a q range whose
 * pairs are not all held.  With a pair subset and no separate HF integrals, hf_fock returns the
 * partial Fock matrix of the q range (exchange over k' = k + q of those q; the direct and
 * Madelung terms on the context whose range holds q = 0), so that the ranks' matrices add up to
 * the full one.  gw_sigma_vjp needs the full pair set.  gb200_set_integrals or
 * gb200_set_integrals_device (GW) go back to the full pair set. */
int gb200_set_integrals_pairs(gb200_context* ctx, const double* V_pairs, const int64_t* pair_ids, int64_t count,
                              int on_device, void* stream);

/* The "extrapolate" q -> 0 treatment of the GW self-energy (q0_treatment, common_defs.h;
 * mbpt_q0_utils_t.cpp:11-178, call sites gw_cpu_kernel.cpp:58-64,267-270): with AqQ
 * [nk][NQ] (complex, the AqQ dataset of AqQ.h5) and q_abs [nk] (|q|), every gw_sigma call
 * collects eps_inv(i Omega_n, q) = conj(A_q) P(i Omega_n, q) A_q, extrapolates its real part to
 * q -> 0 with a quadratic fit over the distinct |q| in (0, 1], takes it to tau, and adds
 * -madelung eps_inv(tau) S G(tau) S to Sigma (S from gb200_dyson_set_hamiltonian; spinor
 * blocks with S_aa for two-component input).  Needs the full q range in one context.
 * AqQ = NULL switches the correction off. */
int gb200_set_q0_correction(gb200_context* ctx, const double* AqQ, const double* q_abs, double madelung);

/* Contraction precision (GB200_PREC_*) and, for GB200_PREC_SPLIT, the number
 * of INT8 slices per operand (2..8). */
int gb200_set_precision(gb200_context* ctx, int mode, int slices);
/* Slices per contraction under GB200_PREC_SPLIT: slices6[0..2] for the polarization contractions
 * (P0_contraction, gw_cpu_kernel.cpp:200-215, in three GEMM stages) and slices6[3..5] for the
 * self-energy ones (selfenergy_contraction, :359-373); 0 keeps the count of gb200_set_precision,
 * NULL resets all six to 0.  No counterpart in the reference (which runs FP64). */
int gb200_set_contraction_slices(gb200_context* ctx, const int* slices6);

/* Bytes the blocked intermediates of one call may use (the k-block buffers of the GW self-energy
 * and its adjoint, the exchange intermediates of the Fock build); 0 (the default) takes a share of
 * the free device memory at the call.  For several contexts sharing one GPU.  The reference sizes
 * its buffers per MPI rank instead (gw_cpu_kernel.cpp:74-134); no counterpart. */
int gb200_set_memory_budget(gb200_context* ctx, double bytes);

/* GW self-energy: Sigma(tau,k) from G(tau,k), both [nts, ns, nk, nso, nso].
 * Replaces gw_cpu_kernel::solve (gw_cpu_kernel.cpp:31-72): Sigma is zeroed,
 * accumulated over q and divided by nk. */
int gb200_gw_sigma(gb200_context* ctx, const double* G, double* Sigma);
int gb200_gw_sigma_device(gb200_context* ctx, const double* G_dev, double* Sigma_dev, void* stream);

/* Vector-Jacobian product of the GW self-energy (FP64).  With L = Re sum conj(Sb) Sigma(G, V):
 * Gb = dL/dG [nts, ns, nk, nso, nso] and, when Vb is not NULL, Vb = dL/dV for the half-stored GW
 * integrals [nk(nk+1)/2, NQ, nao, nao] (the layout gb200_set_integrals takes), so that
 * dL = Re sum conj(Gb) dG + Re sum conj(Vb) dV for all complex dG, dV.  The reference computes
 * no derivatives: this is the adjoint of gw_cpu_kernel::solve (gw_cpu_kernel.cpp:31-72), for
 * gradients of GW functionals.  Scalar (non-two-component) input without the q -> 0 correction;
 * P0 and W of every q are recomputed in FP64 rather than stored.  Needs one full-pair-set
 * accumulator (nk^2 NQ nao^2 complex) on the device when Vb is requested. */
int gb200_gw_sigma_vjp(gb200_context* ctx, const double* G, const double* Sb, double* Gb, double* Vb);
int gb200_gw_sigma_vjp_device(gb200_context* ctx, const double* G_dev, const double* Sb_dev, double* Gb_dev,
                              double* Vb_dev, void* stream);

/* Hartree-Fock Fock matrix F [ns, nk, nso, nso] from the density matrix dm
 * and overlap S (same shape).  Replaces hf_scalar_cpu_kernel::solve
 * (hf_cpu_kernels.cpp:25-146) and, for nso = 2 nao, hf_x2c_cpu_kernel::solve
 * (:148-279); dm = spin_prefactor * G(beta) as in hf_solver::solve
 * (hf_solver.cpp:9-16). */
int gb200_hf_fock(gb200_context* ctx, const double* dm, const double* S, double madelung, double* F);
int gb200_hf_fock_device(gb200_context* ctx, const double* dm_dev, const double* S_dev, double madelung,
                         double* F_dev, void* stream);

/* The same Fock matrix as gb200_hf_fock_device, for callers that cannot
 * allocate device memory while they run: hosts whose memory pool already
 * holds the free HBM, or that must avoid the device-wide synchronisation of
 * cudaMalloc/cudaFree.  No counterpart in the reference.  It needs no context
 * and calls no allocating routine: the caller passes the dimensions (dims->nk,
 * nao, ns, NQ are read; dims->nso must be 0 or nao, since two-component input
 * is rejected with GB200_ERR_INVALID), the full-storage integrals V_dev [nk][nk][NQ][nao][nao]
 * (complex128, pair (k,k') at ((k*nk + k')*NQ)*nao*nao), dm_dev, S_dev and
 * F_dev [ns][nk][nao][nao], and a stream (NULL = legacy default stream).
 * Working memory is one fixed 64 MiB device array inside the library, which
 * every GPU that loads the library holds until the process exits.  Sizes whose
 * workspace, 16 * (ns*nk*nao^2 + max(ns*NQ*nao^2, ns*nk*nao^2)) bytes plus small
 * tables, does not fit are rejected with GB200_ERR_INVALID and a message
 * readable through gb200_last_error(NULL).  Each call looks up that array's
 * address for the current device and context; while `stream` is being captured
 * it reuses the address an earlier call in the same context found, so make the
 * first call in a context before any stream capture.  Every call shares the
 * array and its contents stay from the last call: calls that overlap on the GPU
 * (different streams or host threads) race.  The call is asynchronous on
 * `stream`. */
int gb200_hf_fock_noalloc(const gb200_dims* dims, const double* V_dev, const double* dm_dev, const double* S_dev,
                          double madelung, double* F_dev, void* stream);

/* Dyson step (dyson.cpp).  H and S: [ns, nk, nso, nso]. */
int gb200_dyson_set_hamiltonian(gb200_context* ctx, const double* H, const double* S);
/* find_mu (dyson.cpp:101-174): bracket with step 0.5 then bisection to `tol`. */
int gb200_dyson_find_mu(gb200_context* ctx, const double* Sigma1, const double* Sigma_tau, double mu0,
                        double nel_target, double tol, double* mu_out, double* nel_out);
/* compute_G (dyson.cpp:238-288): hermitizes Sigma1 and Sigma_tau in the
 * caller's buffers as the reference does, writes G_tau [nts, ns, nk, nso, nso]. */
int gb200_dyson_compute_G(gb200_context* ctx, double* Sigma1, double* Sigma_tau, double mu, double* G);
/* Electron count n(mu) for given self-energies (compute_number_of_electrons, dyson.cpp:72-99). */
int gb200_dyson_electrons(gb200_context* ctx, const double* Sigma1, const double* Sigma_tau, double mu,
                          double* nel_out);
/* (E_1b, E_HF, E_corr) of compute_energy (common_utils.cpp:5-55). */
int gb200_energy(gb200_context* ctx, const double* G, const double* Sigma1, const double* Sigma_tau,
                 double* e_out3);

/* One self-consistency iteration on device buffers, the sequence mbpt.exe
 * runs per iteration (mbpt_run.h:199-209, dyson.cpp:290-317):
 *   Sigma1 = HF(dm(G)), Sigma_tau = GW(G), mu = find_mu (if nel_target > 0),
 *   G <- compute_G, energies.
 * G_dev is overwritten with the new Green's function. */
int gb200_iteration_device(gb200_context* ctx, double* G_dev, double* Sigma1_dev, double* Sigma_dev,
                           double madelung, double nel_target, double tol, double* mu_inout, double* e_out3,
                           void* stream);

/* Dyson step on device buffers: find_mu (if nel_target > 0, dyson.cpp:101-174) then
 * compute_G (dyson.cpp:238-288); Sigma1/Sigma are hermitized in place. */
int gb200_dyson_solve_device(gb200_context* ctx, double* Sigma1_dev, double* Sigma_dev, double nel_target, double tol,
                             double* mu_inout, double* G_dev, void* stream);
/* compute_energy (common_utils.cpp:5-55) on device buffers. */
int gb200_energy_device(gb200_context* ctx, const double* G_dev, const double* Sigma1_dev, const double* Sigma_dev,
                        double* e_out3, void* stream);

/* Kernel statistics for measurement: gb200_stats_enable(ctx, 1) starts timing every
 * launch of the tensor-core contraction kernel with CUDA events on its stream;
 * gb200_stats_read returns the library's total kernel-launch count (process wide),
 * and for the contraction kernel its launches, summed device time (ms) and summed
 * FP64-equivalent complex flops (8 per complex multiply-add). */
int gb200_stats_enable(gb200_context* ctx, int on);
int gb200_stats_read(gb200_context* ctx, long long* launches_total, long long* tc_launches, double* tc_ms,
                     double* tc_alg_flops);

/* Select the engine that multiplies the INT8 slice planes of GB200_PREC_SPLIT:
 * 0 = tcgen05 tensor cores (default), 1 = CUDA-core validation engine that
 * forms the same INT32 diagonal sums from the same planes (results must agree
 * bit for bit).  No counterpart in the reference (its kernels are FP64 only). */
int gb200_set_split_engine(gb200_context* ctx, int engine);

/* Timing of the last gb200_gw_sigma* call by stage, milliseconds, CUDA events:
 * out[0] P0, out[1] W solve and transforms, out[2] Sigma, out[3] total. */
int gb200_last_timings(const gb200_context* ctx, float* out4);

#ifdef __cplusplus
}
#endif

#endif /* GB200_H */
