/*
 * stkfmm_b200.h -- C ABI of the B200 (sm_100a) STKFMM kernel-evaluation path.
 *
 * Drop-in boundary for STKFMM's direct kernel-evaluation hot path:
 *   - the Stk3DFMM_* handle API of Lib/include/STKFMM/STKFMM.h:5-36 and
 *     Lib/src/Stk3DFMM-c.cpp:5-67 (same names, argument order and
 *     accumulate-into-output semantics; every call returns a status code
 *     instead of printing and calling exit(1));
 *   - STKFMM::evaluateKernel (Lib/include/STKFMM/STKFMM.hpp:108-110,
 *     Lib/src/STKFMM.cpp:88-99, Lib/src/FMMData.cpp:252-283), which the
 *     reference C ABI never exported;
 *   - list-level P2P entry points over device-resident, leaf-sorted arrays, the
 *     unit of work PVFMM's PtFMM_Evaluate performs per (target box, source box)
 *     pair through Kernel<T>::ker_poten (Lib/src/FMMData.cpp:198, 280-281);
 *   - ker_poten-signature shims, one per STKFMM micro-kernel, that a PVFMM build
 *     could register in place of the CPU uKerEval bodies.
 *
 * Host pointers are plain double arrays owned by the caller (AoS xyz, AoS
 * values), as in the reference.  Device pointers are only taken by the
 * *_device / *_lists entry points and are never freed by the library.
 * The library fails loudly (STK_ERR_NO_DEVICE) when no CUDA device is present:
 * there is no CPU fallback.
 */
/* One guard per inclusion site: stkfmm_b200.hpp also includes this header inside
 * namespace stkfmm::capi (with STKFMM_B200_IN_NAMESPACE defined), so that its C++
 * classes can share their names with these C handle types. */
#if (defined(STKFMM_B200_IN_NAMESPACE) && !defined(STKFMM_B200_NS_H_)) || \
    (!defined(STKFMM_B200_IN_NAMESPACE) && !defined(STKFMM_B200_H_))
#ifdef STKFMM_B200_IN_NAMESPACE
#define STKFMM_B200_NS_H_
#else
#define STKFMM_B200_H_
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum stk_status {
    STK_OK = 0,
    STK_ERR_INVALID_ARG = 1,  /* null pointer, negative size, bad enum value            */
    STK_ERR_KERNEL = 2,       /* kernel not activated / no such sub-kernel (STKFMM.cpp:53-55) */
    STK_ERR_STATE = 3,        /* call order: set_points / setup_tree missing              */
    STK_ERR_SIZE = 4,         /* point / value counts disagree (FMMData.cpp:184-195)      */
    STK_ERR_CUDA = 5,         /* a CUDA runtime call failed                               */
    STK_ERR_NO_DEVICE = 6,    /* no CUDA device: this library has no CPU path             */
    STK_ERR_OUT_OF_BOX = 7,   /* a point lies outside the FMM box on a free axis          */
    STK_ERR_NOT_SUPPORTED = 8 /* kernel or feature not provided by this library           */
};

/* ---- enums of Lib/include/STKFMM/STKFMM_common.hpp ---------------------- */
/* PAXIS (STKFMM_common.hpp:29-34) */
enum stk_paxis { STK_PAXIS_NONE = 0, STK_PAXIS_PX = 1, STK_PAXIS_PXY = 2, STK_PAXIS_PXYZ = 3 };
/* PPKERNEL (STKFMM_common.hpp:40-44) */
enum stk_ppkernel { STK_SLS2T = 1, STK_DLS2T = 2, STK_L2T = 4 };
/* KERNEL (STKFMM_common.hpp:46-62) */
enum stk_kernel {
    STK_LapPGrad = 1,
    STK_LapPGradGrad = 2,
    STK_LapQPGradGrad = 4,
    STK_Stokes = 8,
    STK_RPY = 16,
    STK_StokesRegVel = 32,
    STK_StokesRegVelOmega = 64,
    STK_PVel = 128,
    STK_PVelGrad = 256,
    STK_PVelLaplacian = 512,
    STK_Traction = 1024
};

/* Arithmetic of the P2P kernels.  FP64: plain double.  MIXED: FP64
 * centre-relative displacement, FP32 kernel tensor (MUFU rsqrt + 1 Newton
 * step), Kahan-compensated FP32 accumulation per target. */
enum stk_precision { STK_FP64 = 0, STK_MIXED = 1 };

/* Micro-kernels: one STKFMM uKerEval body each (sources -> targets dims). */
enum stk_ukernel {
    STK_UK_LAPLACE_P = 0,           /* 1 -> 1   LaplaceLayerKernel.hpp:41-65                */
    STK_UK_LAPLACE_PGRAD = 1,       /* 1 -> 4   LaplaceLayerKernel.hpp:67-96                */
    STK_UK_LAPLACE_DIPOLEP = 2,     /* 3 -> 1   LaplaceLayerKernel.hpp:98-113               */
    STK_UK_LAPLACE_DIPOLEPGRAD = 3, /* 3 -> 4   LaplaceLayerKernel.hpp:115-136              */
    STK_UK_STOKES_VEL = 4,          /* 3 -> 3   PVFMM stokes_vel, StokesLayerKernel.hpp:39-42 */
    STK_UK_RPY_U = 5,               /* 4 -> 3   RPYKernel.hpp:17-45                         */
    STK_UK_RPY_ULAPU = 6,           /* 4 -> 6   RPYKernel.hpp:52-90                         */
    STK_UK_STK_ULAPU = 7,           /* 3 -> 6   RPYKernel.hpp:97-129                        */
    STK_UK_STOKES_REGVEL = 8,       /* 4 -> 3   StokesRegSingleLayerKernel.hpp:17-41        */
    STK_UK_STOKES_PVEL = 9,         /* 4 -> 4   StokesSingleLayerKernel.hpp:27-47           */
    STK_UK_STOKES_DOUBLEPVEL = 10,  /* 9 -> 4   StokesDoubleLayerKernel.hpp:25-57           */
    STK_UK_LAPLACE_SLDL_PGRAD = 11, /* 1+3 -> 4 laplace_pgrad + laplace_dipolepgrad at one point */
    STK_UK_STOKES_SLDL_PVEL = 12,   /* 4+9 -> 4 stokes_pvel + stokes_doublepvel at one point     */
    /* Adjoint of stokes_regvel (no reference counterpart).  Both read 3 or 4
     * values per OUTPUT point (stk_ukernel_aux_dim) and evaluate at the
     * displacement (output point - input point):
     *   ADJ_SRC: outputs = forward sources with values (f, eps), inputs = forward
     *            targets with values w = dL/du  ->  (dL/df 3, dL/deps 1, dL/dx_src 3)
     *   ADJ_TRG: outputs = forward targets with values w, inputs = forward sources
     *            with values (f, eps)  ->  dL/dx_trg 3 */
    STK_UK_REGVEL_ADJ_SRC = 13,     /* 3 -> 7, 4 values per output point */
    STK_UK_REGVEL_ADJ_TRG = 14,     /* 4 -> 3, 3 values per output point */
    STK_UK_LAPLACE_SLDL_P = 15,     /* 1+3 -> 1 laplace_p + laplace_dipolep at one point */
    /* outputs (p, grad p 3, Hessian xx xy xz yy yz zz) */
    STK_UK_LAPLACE_PGRADGRAD = 16,       /* 1 -> 10  LaplaceLayerKernel.hpp:138-166 */
    STK_UK_LAPLACE_DIPOLEPGRADGRAD = 17, /* 3 -> 10  LaplaceLayerKernel.hpp:168-200 */
    STK_UK_LAPLACE_QUADP = 18,           /* 9 -> 1   LaplaceLayerKernel.hpp:202-232 (S row-major) */
    STK_UK_LAPLACE_QUADPGRADGRAD = 19,   /* 9 -> 10  LaplaceLayerKernel.hpp:234-301 */
    /* Stokes derivatives: (p, u 3, grad p 3, grad u 9 as du_i/dx_j at 7 + 3i + j),
     * (p, u 3, lap u 3), traction 3x3 row-major */
    STK_UK_STOKES_PVELGRAD = 20,         /* 4 -> 16  StokesSingleLayerKernel.hpp:54-111 */
    STK_UK_STOKES_DOUBLEPVELGRAD = 21,   /* 9 -> 16  StokesDoubleLayerKernel.hpp:64-143 */
    STK_UK_STOKES_PVELLAPLACIAN = 22,    /* 4 -> 7   StokesSingleLayerKernel.hpp:118-155 */
    STK_UK_STOKES_DOUBLELAPLACIAN = 23,  /* 9 -> 7   StokesDoubleLayerKernel.hpp:150-206 */
    STK_UK_STOKES_TRACTION = 24,         /* 4 -> 9   StokesSingleLayerKernel.hpp:162-199 */
    STK_UK_STOKES_DOUBLETRACTION = 25,   /* 9 -> 9   StokesDoubleLayerKernel.hpp:213-276 */
    /* regularized force + torque (f, t, eps) and the point-force (u, omega) kernel */
    STK_UK_STOKES_REGFTVEL = 26,         /* 7 -> 3   StokesRegSingleLayerKernel.hpp:48-89   */
    STK_UK_STOKES_REGFTVELOMEGA = 27,    /* 7 -> 6   StokesRegSingleLayerKernel.hpp:96-151  */
    STK_UK_STOKES_VELOMEGA = 28          /* 3 -> 6   StokesRegSingleLayerKernel.hpp:158-203 */
};

/* ---- kernel descriptors --------------------------------------------------- */
const char *stk_status_string(int status);
/* dims = {kdimSL, kdimDL, kdimTrg}; replaces getKernelDimension (Lib/src/STKFMM.cpp:33-40) */
int stk_get_kernel_dimension(unsigned kernel, int *dims);
/* PVFMM kernel name of the S2T kernel (getKernelName, Lib/src/STKFMM.cpp:42-47) */
const char *stk_get_kernel_name(unsigned kernel);
/* Box scaling of a kernel (host only): the factors by which the single-layer
 * values sl[kdimSL], the double-layer values dl[kdimDL] and the results
 * trg[kdimTrg] are multiplied around the unit-box FMM for a box with scale
 * factor sf = 1 / length (FMMData::scaleSrc / scaleTrg, FMMData.cpp:285-470). */
int stk_kernel_scaling(unsigned kernel, double sf, double *sl, double *dl, double *trg);
/* micro-kernel that fills a PVFMM slot of a kernel: slot 0 s2t SL, 1 s2t DL,
 * 2 s2m SL, 3 s2m DL, 4 m2m/m2l/l2l, 5 m2t, 6 l2t, 7 s2l SL, 8 s2l DL;
 * -1 when the slot is empty.  Mirrors the BuildKernel compositions, e.g.
 * RPYKernel.hpp:137-154, LaplaceLayerKernel.hpp:314-326. */
int stk_kernel_slot(unsigned kernel, int slot);
int stk_ukernel_dims(int ukernel, int *sdim, int *tdim);
/* values per output point a micro-kernel reads (0 for all but the adjoint kernels) */
int stk_ukernel_aux_dim(int ukernel);
int stk_device_count(void);
/* Throughput probes of the running GPU (no reference counterpart; roofline
 * denominators of the P2P kernels): out[0] FP32 TFLOP/s (FMA = 2 flops),
 * out[1] FP64 TFLOP/s, out[2] MUFU rsqrt Gop/s, out[3] SM clock MHz seen by the
 * probe, out[4] SM count, out[5] packed FP32 (fma.rn.f32x2) TFLOP/s. */
int stk_measure_peaks(double *out);

/* ---- direct sum (STKFMM::evaluateKernel) --------------------------------- */
/* trg_value += K(trg - src) src_value over all pairs, host arrays, raw
 * coordinates (no box scaling), accumulate.  ppkernel picks the k_s2t SL
 * (SLS2T), k_s2t DL (DLS2T) or k_l2t (L2T) sub-kernel as FMMData.cpp:261-268. */
int stk_evaluate_kernel(unsigned kernel, unsigned ppkernel, int nsrc, const double *src_coord,
                        const double *src_value, int ntrg, const double *trg_coord, double *trg_value,
                        int precision);
/* Same on device pointers and a caller's cudaStream_t (passed as void *).  The
 * device-pointer entry points (this one, stk_ukernel_direct_device[_aux],
 * stk_p2p_lists[_aux]) queue their work on `stream` and return without a host
 * wait; the calling thread's scratch buffers are ordered across calls by an
 * event (a later call's stream waits for the earlier call's work). */
int stk_evaluate_kernel_device(unsigned kernel, unsigned ppkernel, int nsrc, const double *d_src_coord,
                               const double *d_src_value, int ntrg, const double *d_trg_coord,
                               double *d_trg_value, int precision, void *stream);
/* Direct sum of one micro-kernel on device pointers. */
int stk_ukernel_direct_device(int ukernel, int nsrc, const double *d_src_coord, const double *d_src_value,
                              int ntrg, const double *d_trg_coord, double *d_trg_value, int precision,
                              void *stream);
/* Direct sum of a micro-kernel that reads values per output point (the adjoint
 * kernels): d_trg_aux holds stk_ukernel_aux_dim(ukernel) doubles per target. */
int stk_ukernel_direct_aux_device(int ukernel, int nsrc, const double *d_src_coord, const double *d_src_value,
                                  int ntrg, const double *d_trg_coord, const double *d_trg_aux, double *d_trg_value,
                                  int precision, void *stream);
/* The same direct sum for callers that cannot allocate device memory while they
 * run: frameworks whose own caching allocator owns the device (memory taken
 * behind its back can make it fail), programs that keep several streams busy
 * and cannot afford the device-wide synchronisation of cudaMalloc/cudaFree,
 * hosts that forbid run-time allocation.  No reference counterpart.
 * It calls no cudaMalloc/cudaFree: all scratch lives in one fixed 8 MiB array
 * that the library reserves on every GPU where it is loaded.  Sizes whose
 * scratch (work list + nsrc packed source records) exceeds 8 MiB are refused
 * with STK_ERR_SIZE (about 130k sources for 8-double records).  It takes every
 * micro-kernel stk_ukernel_direct_device takes without per-target values; the
 * adjoint ids (13, 14) are refused with STK_ERR_INVALID_ARG.  The first call on
 * a device looks the array up (cudaGetSymbolAddress) and the first call of each
 * (ukernel, precision) pair runs a one-time occupancy query; make those calls
 * before any stream capture.  Not to be used again after a cudaDeviceReset of
 * the device.  Work is queued on `stream` without a host wait.  All calls share
 * the array: calls that overlap on the GPU race; outputs accumulate. */
int stk_ukernel_direct_device_noalloc(int ukernel, int nsrc, const double *d_src_coord, const double *d_src_value,
                                      int ntrg, const double *d_trg_coord, double *d_trg_value, int precision,
                                      void *stream);

/* ---- list-level P2P ---------------------------------------------------------
 * One micro-kernel over an explicit interaction list (device pointers):
 *   target box b owns targets [trg_begin[b], trg_end[b]) of d_trg_coord / d_trg_value;
 *   source box s owns sources [src_begin[s], src_end[s]) of d_src_coord / d_src_value;
 *   list_off[b] .. list_off[b+1]-1 index list_ent, each entry
 *   (source box << 5) | (sx+1) + 3(sy+1) + 9(sz+1), the source image shifted by
 *   (sx, sy, sz) * period.  Index arrays are host arrays (the library builds the
 *   cost-sorted work list from them).  Outputs accumulate. */
int stk_p2p_lists(int ukernel, int precision, int n_trg_box, const int *trg_begin, const int *trg_end,
                  const int *list_off, const int *list_ent, int n_src_box, const int *src_begin,
                  const int *src_end, int nsrc, const double *d_src_coord, const double *d_src_value, int ntrg,
                  const double *d_trg_coord, double *d_trg_value, double period, void *stream);
/* The same for micro-kernels with per-output-point values (the adjoint kernels). */
int stk_p2p_lists_aux(int ukernel, int precision, int n_trg_box, const int *trg_begin, const int *trg_end,
                      const int *list_off, const int *list_ent, int n_src_box, const int *src_begin,
                      const int *src_end, int nsrc, const double *d_src_coord, const double *d_src_value, int ntrg,
                      const double *d_trg_coord, const double *d_trg_aux, double *d_trg_value, double period,
                      void *stream);

/* ---- tensor-core GEMM of the mixed-precision M2L ------------------------------
 * No reference counterpart (the reference's far field is PVFMM's FP64 BLAS).
 * C[m + n ldc] (beta 0: =, 1: +=) sum_k A[m lda + k] B[n ldb + k] for m < M,
 * n < N: FP32 in and out, computed on the sm_100a tensor cores (tcgen05, TF32)
 * to FP32 accuracy: each operand split into a TF32 high part and an FP32
 * remainder (3 products), every 32-wide K-block accumulated on its own and
 * drained into FP32 registers.  Device pointers; the call copies the operands
 * into padded, split scratch that it allocates, and waits for the result.
 * STK_ERR_NOT_SUPPORTED off sm_100. */
int stk_gemm_3xtf32(int M, int N, int K, const float *d_A, int lda, const float *d_B, int ldb, float *d_C, int ldc,
                    int beta, void *stream);

/* ---- reusable asynchronous list plan -----------------------------------------
 * Replaces, for a list evaluated many times, the per-(target box, source box)
 * ker_poten calls that PVFMM's list loops make at every evaluation
 * (PtFMM_Evaluate, Lib/src/FMMData.cpp:198).  stk_p2p_plan_create validates a
 * CSR list (the layout of stk_p2p_lists, host arrays), builds its cost-sorted
 * work items and uploads list and items into device memory owned by the plan
 * (on the current device); *status gets STK_OK or the error, NULL is returned on
 * error.  stk_p2p_plan_execute queues one micro-kernel over the plan's list on
 * `stream` and returns without a host wait; outputs accumulate.  The plan's
 * scratch (the packed source records and the work counter) is shared by its
 * executions: executions of one plan must be ordered (one stream, or the caller
 * synchronises between streams).  The first execution with a larger record
 * stride allocates (and synchronises the device).  d_trg_aux: per-target values
 * of the adjoint micro-kernels (stk_ukernel_aux_dim), else NULL.
 * stk_p2p_plan_destroy waits for the device before freeing. */
typedef struct stk_p2p_plan stk_p2p_plan;
stk_p2p_plan *stk_p2p_plan_create(int n_trg_box, const int *trg_begin, const int *trg_end, const int *list_off,
                                  const int *list_ent, int n_src_box, const int *src_begin, const int *src_end,
                                  int nsrc, int ntrg, double period, int *status);
int stk_p2p_plan_execute(stk_p2p_plan *plan, int ukernel, int precision, const double *d_src_coord,
                         const double *d_src_value, const double *d_trg_coord, const double *d_trg_aux,
                         double *d_trg_value, void *stream);
/* (target, source point) pairs of the plan's list */
long long stk_p2p_plan_pairs(const stk_p2p_plan *plan);
void stk_p2p_plan_destroy(stk_p2p_plan *plan);

/* ---- Stk3DFMM handle (Lib/include/STKFMM/STKFMM.h, Lib/src/Stk3DFMM-c.cpp) -- */
typedef struct Stk3DFMM Stk3DFMM;
/* Stk3DFMM-c.cpp:5-7; returns NULL on invalid arguments or when no device */
Stk3DFMM *Stk3DFMM_create(int mult_order, int max_pts, int pbc, unsigned kernelComb);
void Stk3DFMM_destroy(Stk3DFMM *fmm);
/* Stk3DFMM-c.cpp:13-16 */
int Stk3DFMM_set_points(Stk3DFMM *fmm, const int nSL, double *src_SL_coord, const int nTrg, double *trg_coord,
                        const int nDL, double *src_DL_coord);
/* Stk3DFMM-c.cpp:18-20 (not declared in the reference header) */
int Stk3DFMM_get_kernel_dimension(unsigned kernel, int *dims);
/* Stk3DFMM-c.cpp:22 */
int Stk3DFMM_set_box(Stk3DFMM *fmm, double *origin, double len);
/* Stk3DFMM-c.cpp:24 */
int Stk3DFMM_setup_tree(Stk3DFMM *fmm, unsigned kernel);
/* Stk3DFMM-c.cpp:26 (not declared in the reference header) */
int Stk3DFMM_clear_fmm(Stk3DFMM *fmm, unsigned kernel);
/* Stk3DFMM-c.cpp:28-31: trg_value += FMM(sources): U-list near field plus the
 * KIFMM far field, for every kernel of STKFMM_common.hpp:46-62 (LapPGrad,
 * LapPGradGrad, LapQPGradGrad, Stokes, RPY, StokesRegVel, StokesRegVelOmega,
 * PVel, PVelGrad, PVelLaplacian, Traction) in free space, PX, PXY and PXYZ.
 * Triply periodic potentials / pressures / mean velocities carry a constant
 * per component (drift) set by the equivalent density, as in the reference. */
int Stk3DFMM_evaluate_fmm(Stk3DFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value, const int nTrg,
                          double *trg_value, const int nDL, double *src_DL_value);
/* Stk3DFMM-c.cpp:33-35 */
int Stk3DFMM_show_active_kernels(Stk3DFMM *fmm);

/* additions with no reference C counterpart */
/* STKFMM::evaluateKernel through the handle (STKFMM.cpp:88-99) */
int Stk3DFMM_evaluate_kernel(Stk3DFMM *fmm, unsigned kernel, int nThreads, unsigned p2p, int nSrc,
                             double *srcCoord, double *srcValue, int nTrg, double *trgCoord, double *trgValue);
/* choose FP64 or MIXED for the P2P kernels of this handle (default FP64) */
int Stk3DFMM_set_precision(Stk3DFMM *fmm, int precision);
/* Multi-GPU sharding of one problem: this handle evaluates only shard `rank` of
 * `nranks` of the target-side work (near-field P2P, L2T, M2T), dealt by cost;
 * the upward pass, S2L and M2L are computed in full on every shard.  The sum of
 * all shards' evaluate_near / evaluate_fmm outputs (e.g. an all-reduce) is the
 * unsharded result.  Takes effect at the next setup_tree (default 0 of 1). */
int Stk3DFMM_set_shard(Stk3DFMM *fmm, int rank, int nranks);
/* Collective of a sharded handle: sum the n doubles at d_buf (device memory of the
 * handle's GPU) in place over the ranks of the shard group, ordered after the work
 * already queued on `stream` (a cudaStream_t) and before the work queued after the
 * call returns.  Returns 0 on success.  No reference counterpart: the reference
 * distributes its FMM with MPI inside PVFMM (Lib/src/FMMData.cpp:63).  With a
 * collective set and set_shard(rank, n > 1), evaluate_fmm also splits the far
 * field: each rank runs the M2L and S2L of its share of the target nodes (nodes
 * of complete levels by parity type, the others by cost) and the ranks' downward
 * equivalent densities are summed with one call of fn (nodes x n_surface x kdim
 * doubles) before the L2L.  Every rank then holds the whole downward pass; the
 * near field, L2T and M2T stay split as set_shard describes, so the sum of the
 * ranks' target outputs is still the unsharded result.  fn = NULL: the far field
 * is not split (each rank computes all of it).  Takes effect at the next
 * setup_tree. */
typedef int (*stk_allreduce_fn)(double *d_buf, long long n, void *stream, void *user);
int Stk3DFMM_set_allreduce(Stk3DFMM *fmm, stk_allreduce_fn fn, void *user);

/* The periodic far field, the reference's enableFF constructor argument
 * (STKFMM.hpp:199-200, FMMData.cpp:83-89; its C ABI always passes true).  enable = 0:
 * no far-image operator and no periodizeFMM correction, so a periodic sum stops
 * at the images within two cells of the unit cell on each periodic axis, the
 * images PVFMM's periodic lists reach.  Takes effect at the next setup_tree
 * (default 1).  No effect in free space. */
int Stk3DFMM_set_far_field(Stk3DFMM *fmm, int enable);
/* Near-field (U-list S2T) part of evaluate_fmm only, on the tree of setup_tree:
 * trg_value += sum over U-list leaf pairs, in the caller's coordinates/units. */
int Stk3DFMM_evaluate_near(Stk3DFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value, const int nTrg,
                           double *trg_value, const int nDL, double *src_DL_value);
/* Same on device buffers in the caller's order (values as given, unit box only:
 * STK_ERR_NOT_SUPPORTED otherwise), queued on `stream` (a cudaStream_t, or null for
 * the handle's stream) without a host synchronisation. */
int Stk3DFMM_evaluate_near_device(Stk3DFMM *fmm, unsigned kernel, const double *d_src_SL_value, double *d_trg_value,
                                  const double *d_src_DL_value, void *stream);
/* evaluate_fmm on device buffers in the caller's order (values as given, unit
 * box only: STK_ERR_NOT_SUPPORTED otherwise), queued on `stream` without a host
 * synchronisation: d_trg_value += near field + KIFMM far field.  The first call
 * after setup_tree builds the far-field operators and synchronises. */
int Stk3DFMM_evaluate_fmm_device(Stk3DFMM *fmm, unsigned kernel, const double *d_src_SL_value, double *d_trg_value,
                                 const double *d_src_DL_value, void *stream);
/* Device time (ms, CUDA events on the launching stream) of the kernel launches
 * of the last near-field or FMM evaluation of `kernel`. */
int Stk3DFMM_last_kernel_ms(Stk3DFMM *fmm, unsigned kernel, float *ms);
/* Device time (ms) of each phase of the last evaluation of `kernel`: ms[0] U-list
 * P2P, [1] S2M + check-to-equivalent solve, [2] M2M, [3] M2L, [4] S2L + solve,
 * [5] L2L, [6] L2T, [7] M2T (W list); [1..7] are 0 after a near-field-only call. */
int Stk3DFMM_last_phase_ms(Stk3DFMM *fmm, unsigned kernel, float *ms);
/* Number of this library's kernels launched by the last evaluation of `kernel`
 * (near-field or FMM; cuBLAS calls of the far field excluded). */
int Stk3DFMM_last_launch_count(Stk3DFMM *fmm, unsigned kernel, int *count);
/* Tree / list statistics of the last setup_tree for `kernel`:
 * out[0] nodes, [1] leaves, [2] depth, [3] U-list entries, [4] U-list SL point pairs,
 * [5] U-list DL point pairs, [6] V entries, [7] W entries, [8] X entries. */
int Stk3DFMM_get_tree_stats(Stk3DFMM *fmm, unsigned kernel, long long *out);
/* Work of one evaluate_fmm of `kernel` (after its first call): out[0] near-field
 * (U list + direct W / X) SL point pairs, [1] DL point pairs, [2] S2M, [3] S2L,
 * [4] M2T, [5] L2T point pairs (sources x check / surface points), [6] M2L node
 * pairs, [7] points per check / equivalent surface, [8] rank of the compressed M2L,
 * [9] kernels of this library launched by the last evaluation (cuBLAS calls excluded). */
int Stk3DFMM_get_fmm_stats(Stk3DFMM *fmm, unsigned kernel, long long *out);
/* Floating-point work of one compressed M2L of `kernel` (after its first evaluate_fmm):
 * out[0] = 4 k r_d per V-list pair at the offsets' true ranks plus the two basis
 * products (4 N k per node), out[1] = the flops the GEMMs execute (ranks padded to
 * multiples of 32, columns to 256-pair chunks). */
int Stk3DFMM_get_m2l_work(Stk3DFMM *fmm, unsigned kernel, double *out);
/* Copy the U-list of the last setup_tree (leaf-sorted indices, same layout as
 * stk_p2p_lists).  Pass null arrays to query sizes: sizes = {n_leaf_boxes, n_entries, nSL, nDL, nTrg}. */
int Stk3DFMM_get_ulist(Stk3DFMM *fmm, unsigned kernel, int *sizes, int *trg_begin, int *trg_end, int *list_off,
                       int *list_ent, int *sl_begin, int *sl_end, int *dl_begin, int *dl_end, int *sl_perm,
                       int *dl_perm, int *trg_perm);

/* ---- StkWallFMM handle (STKFMM.h:19-35, Stk3DFMM-c.cpp:37-67) ---------------
 * Stokeslets (Stokes, 3 values -> u 3) or RPY spheres (RPY, (f, b) -> (u, lap u))
 * above a no-slip wall at z = origin_z; points lie in [o, o+L)^2 x [o_z, o_z+L/2).
 * Each evaluation combines sub-FMMs of the sources and their mirror images
 * (Stokes, LapPGrad, LapPGradGrad; RPY, LapPGradGrad, LapPGrad, LapQPGradGrad),
 * StkWallFMM.cpp:154-292.  Free space, PX or PXY. */
typedef struct StkWallFMM StkWallFMM;
/* Stk3DFMM-c.cpp:37-39; NULL for pbc = PXYZ, without Stokes or RPY in kernelComb,
 * on invalid arguments or when no device */
StkWallFMM *StkWallFMM_create(int mult_order, int max_pts, int pbc, unsigned kernelComb);
/* Stk3DFMM-c.cpp:41-43 */
void StkWallFMM_destroy(StkWallFMM *fmm);
/* Stk3DFMM-c.cpp:45-48; double-layer points are ignored, as in the reference.
 * STK_ERR_OUT_OF_BOX for a point outside [o, o+L)^2 x [o_z, o_z+L/2) on a free axis */
int StkWallFMM_set_points(StkWallFMM *fmm, const int nSL, double *src_SL_coord, const int nTrg, double *trg_coord,
                          const int nDL, double *src_DL_coord);
/* Stk3DFMM-c.cpp:50-52 */
int StkWallFMM_get_kernel_dimension(unsigned kernel, int *dims);
/* Stk3DFMM-c.cpp:54 */
int StkWallFMM_set_box(StkWallFMM *fmm, double *origin, double len);
/* Stk3DFMM-c.cpp:56; STK_ERR_NOT_SUPPORTED for kernels other than Stokes and RPY */
int StkWallFMM_setup_tree(StkWallFMM *fmm, unsigned kernel);
/* Stk3DFMM-c.cpp:58 */
int StkWallFMM_clear_fmm(StkWallFMM *fmm, unsigned kernel);
/* Stk3DFMM-c.cpp:60-63: trg_value += wall FMM(sources) */
int StkWallFMM_evaluate_fmm(StkWallFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value, const int nTrg,
                            double *trg_value, const int nDL, double *src_DL_value);
/* Stk3DFMM-c.cpp:65-67 */
int StkWallFMM_show_active_kernels(StkWallFMM *fmm);
/* additions with no reference C counterpart: P2P precision of the Stokes / RPY
 * sub-FMM (the Laplace sub-FMMs, whose terms cancel near the sources, stay FP64); the
 * evaluation on device buffers in the caller's order queued on `stream` (null: the
 * handle's stream; the first call after setup_tree builds the sub-FMMs' far-field
 * operators and synchronises); device time (ms) of the last evaluation */
int StkWallFMM_set_precision(StkWallFMM *fmm, int precision);
/* Stk3DFMM_set_far_field for every sub-FMM (the reference's StkWallFMM enableFF,
 * STKFMM.hpp:233-234); takes effect at the next setup_tree */
int StkWallFMM_set_far_field(StkWallFMM *fmm, int enable);
int StkWallFMM_evaluate_fmm_device(StkWallFMM *fmm, unsigned kernel, const double *d_src_SL_value,
                                   double *d_trg_value, void *stream);
int StkWallFMM_last_kernel_ms(StkWallFMM *fmm, float *ms);
/* this library's kernels launched by the last evaluation of `kernel` (cuBLAS calls excluded) */
int StkWallFMM_last_launch_count(StkWallFMM *fmm, unsigned kernel, int *count);

/* ---- host-only octree (no CUDA call) ------------------------------------------
 * The tree and KIFMM lists that Stk3DFMM_setup_tree builds, in place of PVFMM's
 * PtFMM_Tree::Initialize / InitFMM_Tree / SetupFMM (FMMData.cpp:107-167).  All
 * coordinates must already lie in [0,1)^3 (scaled and wrapped).  List entries
 * are (node << 5) | shift code, as for stk_p2p_lists. */
/* The reference's public KIFMM surface helper stkfmm::surface (host only,
 * Lib/include/STKFMM/stkfmm_helpers.hpp:46-85): out[3 n] receives the
 * n = 6 (p - 1)^2 + 2 check / equivalent surface points, in the reference's
 * order, on the cube of side alpha 2^-depth with lower corner c[3]. */
int stk_surface(int p, const double *c, double alpha, int depth, double *out);
typedef struct stk_octree stk_octree;
stk_octree *stk_octree_build(const double *tree_pts, int n, int max_pts, int pbc, const double *sl, int nsl,
                             const double *dl, int ndl, const double *trg, int ntrg);
void stk_octree_free(stk_octree *t);
/* The shard assignment behind Stk3DFMM_set_shard (host only): n work items in the
 * given order (largest cost first) are dealt to the least-loaded of nparts parts;
 * owner[i] receives the part of item i. */
int stk_partition_lpt(int n, const double *cost, int nparts, int *owner);
/* out = {nodes, leaves, depth, U entries, V entries, W entries, X entries} */
int stk_octree_sizes(const stk_octree *t, long long *out);
/* per node: level, parent (-1 root), first child (-1 leaf, children contiguous), integer coords (3) */
int stk_octree_nodes(const stk_octree *t, int *level, int *parent, int *first_child, int *ixyz);
/* which: 0 U, 1 V, 2 W, 3 X; off has nodes + 1 entries */
int stk_octree_list(const stk_octree *t, int which, int *off, int *ent);
/* set: 0 SL, 1 DL, 2 targets; perm (sorted position -> caller index), per-node ranges */
int stk_octree_set(const stk_octree *t, int set, int *perm, int *node_begin, int *node_end);
/* owner[node] (0 .. nranks-1): the rank that runs the node's M2L and S2L when
 * Stk3DFMM's far field is split over nranks (Stk3DFMM_set_allreduce); host only. */
int stk_octree_far_owners(const stk_octree *t, int nranks, int *owner);

/* ---- ker_poten-signature shims (pvfmm::Kernel<double>::Ker_t) -----------------
 * void (*)(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg,
 *          int trg_cnt, double *k_out, mem::MemoryManager *mem_mgr)
 * k_out += scaled kernel sum, FP64 on the GPU.  dof must be 1 (the only value
 * STKFMM passes, FMMData.cpp:280-281); mem_mgr is ignored. */
void stk_ker_laplace_p(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                       double *k_out, void *mem_mgr);
void stk_ker_laplace_pgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                           double *k_out, void *mem_mgr);
void stk_ker_laplace_dipolep(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                             double *k_out, void *mem_mgr);
void stk_ker_laplace_dipolepgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                 double *k_out, void *mem_mgr);
void stk_ker_stokes_vel(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                        double *k_out, void *mem_mgr);
void stk_ker_rpy_u(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt, double *k_out,
                   void *mem_mgr);
void stk_ker_rpy_ulapu(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                       double *k_out, void *mem_mgr);
void stk_ker_stk_ulapu(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                       double *k_out, void *mem_mgr);
void stk_ker_stokes_regvel(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                           double *k_out, void *mem_mgr);
void stk_ker_stokes_pvel(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                         double *k_out, void *mem_mgr);
void stk_ker_stokes_doublepvel(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                               double *k_out, void *mem_mgr);
void stk_ker_laplace_pgradgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                               double *k_out, void *mem_mgr);
void stk_ker_laplace_dipolepgradgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg,
                                     int trg_cnt, double *k_out, void *mem_mgr);
void stk_ker_laplace_quadp(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                           double *k_out, void *mem_mgr);
void stk_ker_laplace_quadpgradgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                   double *k_out, void *mem_mgr);
void stk_ker_stokes_pvelgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                             double *k_out, void *mem_mgr);
void stk_ker_stokes_doublepvelgrad(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                   double *k_out, void *mem_mgr);
void stk_ker_stokes_pvellaplacian(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                  double *k_out, void *mem_mgr);
void stk_ker_stokes_doublelaplacian(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                    double *k_out, void *mem_mgr);
void stk_ker_stokes_traction(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                             double *k_out, void *mem_mgr);
void stk_ker_stokes_doubletraction(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                   double *k_out, void *mem_mgr);
void stk_ker_stokes_regftvel(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                             double *k_out, void *mem_mgr);
void stk_ker_stokes_regftvelomega(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                                  double *k_out, void *mem_mgr);
void stk_ker_stokes_velomega(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                             double *k_out, void *mem_mgr);
/* status of the last ker_poten shim call on this thread (they return void) */
int stk_ker_last_status(void);

#ifdef __cplusplus
}
#endif

#endif /* STKFMM_B200_H_ / STKFMM_B200_NS_H_ */
