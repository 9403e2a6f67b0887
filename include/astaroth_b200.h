/*
 * astaroth_b200.h -- entry points this library adds next to the reference
 * interface. None of them has a counterpart in the reference's astaroth.h;
 * existing callers never need them. All are exported with C linkage from the
 * same library as astaroth.h and take plain pointers and sizes.
 */
#pragma once
#include "astaroth.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status and plumbing ------------------------------------------------ */

/* Sticky status word of the device: 0 when every kernel so far completed
 * normally; bit 0 = a bounded wait on a TMA barrier timed out. Reading
 * synchronises the device. */
AcResult acDeviceGetStatus(const Device device, unsigned* status);

/* Clears the status word (after the caller has dealt with a reported
 * failure; the device and its buffers stay usable). Synchronises. */
AcResult acDeviceResetStatus(const Device device);

/* Exercises the failure path of the bounded waits: launches one kernel that
 * waits, with the same bounded wait the solve pipeline uses but a limit of
 * `seconds`, on a barrier phase that nothing completes. The wait gives up,
 * the kernel raises status bit 0 and returns, as a pipeline kernel whose
 * copies never arrived would. Synchronises; returns AC_SUCCESS when the
 * status bit was raised and the device still answers. */
AcResult acDeviceCheckWaitLimit(const Device device, const double seconds);

/* The CUDA stream (cudaStream_t) behind a Stream handle, so a caller can
 * order its own work or CUDA events with the device's. */
AcResult acDeviceGetCudaStream(const Device device, const Stream stream, void** cuda_stream);

/* Number of kernels this device has launched since creation. */
AcResult acDeviceGetLaunchCount(const Device device, unsigned long long* count);

/* Tile configuration of the solve kernel: index into the compiled table,
 * -1 for the built-in default. acDeviceAutoOptimize picks one by timing. */
AcResult acDeviceSetSolveConfig(const Device device, const int config);
AcResult acDeviceGetSolveConfig(const Device device, int* config, int* num_configs);

/* Descriptive name of a solve configuration (tile and pipeline depth). */
const char* acSolveConfigName(const int config);

/* Bytes of device memory held by the device's field blocks. */
AcResult acDeviceGetMemoryFootprint(const Device device, size_t* bytes);

/* ---- whole steps -------------------------------------------------------- */

/* One full RK3 step on `stream`: three times (periodic ghost fill of every
 * field, substep over the whole interior, buffer swap) -- the single-device
 * acNodeIntegrate sequence. Asynchronous. */
AcResult acDeviceIntegrateStep(const Device device, const Stream stream, const AcReal dt);

/* `num_steps` full steps replayed from one captured CUDA graph (the graph is
 * built on first use and rebuilt when dt or the configuration changes).
 * Asynchronous; the buffer roles after the call are as after num_steps calls
 * of acDeviceIntegrateStep. */
AcResult acDeviceIntegrateSteps(const Device device, const Stream stream, const AcReal dt,
                                const int num_steps);

/* ---- steps whose time step is chosen on the device --------------------- */

/* One full RK3 step whose dt is the reference standalone's Courant time step
 * (samples/standalone/simulation.cc:429-436, model/host_timestep.cc:33-60,
 * with the shipped module's LSINK = LBFIELD = 0), evaluated on the device from
 * the current state:
 *   dt = timescale * min(AC_cdt dsmin / (max|u| + sqrt(AC_cs2_sound)),
 *                        AC_cdtv dsmin^2 / max(AC_nu_visc, AC_eta, AC_gamma))
 * with max|u| over the interior (the reduction acDeviceReduceVec(RTYPE_MAX) of
 * uux, uuy, uuz, rounded to AcReal) and dsmin = AC_dsmin, or the smallest of
 * AC_dsx, AC_dsy, AC_dsz where AC_dsmin is unset. The standalone does this on
 * the host with a synchronising reduction each step; here the reduction, the
 * time step and the three substeps are queued on `stream` and nothing returns
 * to the host. The dt used, the accumulated simulated time and the number of
 * such steps are kept on the device (acDeviceGetTimestepRecord). Asynchronous.
 * AC_FAILURE if AC_cdt, AC_cdtv, the spacings or timescale are not positive, or
 * if forcing is enabled (its amplitude depends on dt on the host). The
 * reduction uses the Device's reduction scratch: do not run reductions of the
 * same Device on another stream at the same time. */
AcResult acDeviceIntegrateStepCFL(const Device device, const Stream stream, const AcReal timescale);

/* `num_steps` such steps replayed from one captured CUDA graph (built on first
 * use, rebuilt when the uniforms, the configuration or timescale change). */
AcResult acDeviceIntegrateStepsCFL(const Device device, const Stream stream,
                                   const AcReal timescale, const int num_steps);

/* The time-step record of those steps: dt of the last one, the simulated time
 * (the sum of their dt, from the value acDeviceSetSimulationTime set) and how
 * many were taken. Synchronises `stream`; null pointers are skipped. */
AcResult acDeviceGetTimestepRecord(const Device device, const Stream stream, AcReal* dt,
                                   double* time, unsigned long long* steps);

/* Sets the record's simulated time (and clears its dt and step count).
 * Synchronises `stream`. */
AcResult acDeviceSetSimulationTime(const Device device, const Stream stream, const double time);

/* Step diagnostics folded into the last substep (no counterpart in the
 * reference, whose standalone runs separate reductions after each step,
 * samples/standalone/simulation.cc:250-310). When enabled, every substep 2 over
 * the whole interior (acDeviceIntegrateSubstep, acDeviceIntegrateStep(s), the
 * CFL steps, forced or not) also accumulates, over the state it writes, max,
 * min and sum of |u|^2 and sum of exp(lnrho)^2 in FP64. Until that block
 * changes, acDeviceReduceVec(MAX | MIN | RMS, UUX, UUY, UUZ) and
 * acDeviceReduceScal(RMS_EXP, LNRHO) (and their Double, Node and Legacy forms)
 * return these instead of reading the fields again: the first of them copies
 * all four to the host (one synchronisation), the others return at once. MAX
 * and MIN equal a separate reduction bit for bit; the sums differ from one by
 * their summation order only. Off by default. */
AcResult acDeviceSetStepDiagnostics(const Device device, const int enabled);

/* Enables the helical forcing term at the last substep
 * (acc/mhd_solver/stencil_kernel.ac:611-648,713-717; off in the reference's
 * shipped module). Its parameters are the AC_forcing_* / AC_k_force* /
 * AC_ff_hel_* / AC_kaver uniforms. */
AcResult acDeviceSetForcing(const Device device, const int enabled);

/* Helical forcing parameters of one step: replaces the reference standalone's
 * ForcingParams / generateForcingParams / loadForcingParamsToDevice
 * (samples/standalone/model/host_forcing.h:57-64, host_forcing.cc:287-320,
 * :215-235). */
typedef struct {
    AcReal magnitude;
    AcReal k_force[3];
    AcReal ff_hel_re[3];
    AcReal ff_hel_im[3];
    AcReal phase;
    AcReal kaver;
} AcForcingParams;

/* generateForcingParams with its five random draws given: u[0..2] the
 * wavevector's azimuth, polar angle and length, u[3] the phase, u[4] the angle
 * of e about k, each in [0, 1] (the reference draws them in this order from
 * rand() / RAND_MAX). Reads AC_relhel, AC_forcing_magnitude, AC_kmin, AC_kmax
 * from `info`. */
AcResult acForcingParamsFromUniforms(const AcMeshInfo info, const AcReal u[5],
                                     AcForcingParams* params);

/* The same with the draws from a seeded counter-based generator: *state is
 * the seed on the first call and advances by five draws per call, so a run is
 * reproducible from its seed (the reference's rand() stream is not). */
AcResult acForcingParamsGenerate(const AcMeshInfo info, unsigned long long* state,
                                 AcForcingParams* params);

/* loadForcingParamsToDevice for one Device: loads the AC_forcing_magnitude,
 * AC_forcing_phase, AC_k_force*, AC_ff_hel_* and AC_kaver uniforms. Forcing
 * is applied only while acDeviceSetForcing(device, 1) is in effect. */
AcResult acDeviceLoadForcingParams(const Device device, const Stream stream,
                                   const AcForcingParams params);

/* ---- ensembles ------------------------------------------------------------
 * Many independent meshes (members) of possibly different sizes and
 * parameters on one GPU, advanced together: each substep is ONE ghost-fill
 * launch and ONE persistent solve launch over the tiles of all members, and
 * whole steps replay from a captured CUDA graph. Each member's AcMeshInfo
 * supplies its size and physics (AC_nu_visc, AC_eta, ...); dt is common. */
typedef struct ensemble_s* Ensemble;

AcResult acEnsembleCreate(const int device_id, const int num_members, const AcMeshInfo* configs,
                          Ensemble* ensemble);
AcResult acEnsembleDestroy(Ensemble ensemble);
/* Whole-mesh transfers of one member (mx*my*mz per field, reference order). */
AcResult acEnsembleLoadMember(Ensemble ensemble, const int member, const AcMesh host_mesh);
AcResult acEnsembleStoreMember(Ensemble ensemble, const int member, AcMesh* host_mesh);
/* One RK3 step of every member: 3 x (batched ghost fill, batched substep,
 * swap). Asynchronous on the ensemble's stream. */
AcResult acEnsembleIntegrateStep(Ensemble ensemble, const AcReal dt);
/* num_steps steps replayed from a captured graph (one per buffer parity). */
AcResult acEnsembleIntegrateSteps(Ensemble ensemble, const AcReal dt, const int num_steps);
AcResult acEnsembleSynchronize(Ensemble ensemble);
AcResult acEnsembleGetStatus(Ensemble ensemble, unsigned* status);
AcResult acEnsembleGetCudaStream(Ensemble ensemble, void** cuda_stream);
AcResult acEnsembleGetLaunchCount(Ensemble ensemble, unsigned long long* count);
/* Schedule: tile configuration (index into the compiled table) and the target
 * number of planes per z segment of a task (0 = whole columns). */
AcResult acEnsembleSetSchedule(Ensemble ensemble, const int config, const int segment_planes);
AcResult acEnsembleGetSchedule(Ensemble ensemble, int* config, int* segment_planes);
/* Times every (configuration, segment length) pair on this ensemble and keeps
 * the fastest; results are cached in a text file keyed by the precision and
 * the member sizes (cache_path NULL: $ACB_TUNE_CACHE, else
 * ~/.cache/astaroth_b200/tune.txt). Only the scratch `out` buffers are
 * touched, so the members' states are preserved between whole steps. */
AcResult acEnsembleAutoOptimize(Ensemble ensemble, const char* cache_path);

/* ---- double-precision views (useful in every build; exact in dp) --------- */

/* Loads / stores one whole field (mx*my*mz values, reference index order)
 * from / to a double array. In the mixed build the double is split into the
 * state's float hi part and bfloat16 lo part on load and recombined on store,
 * so a value round trips to about 32 significant bits (24 in hi, 8 more in lo;
 * relative error below 2^-32). */
AcResult acDeviceLoadVertexBufferDouble(const Device device, const Stream stream,
                                        const VertexBufferHandle handle, const double* src);
AcResult acDeviceStoreVertexBufferDouble(const Device device, const Stream stream,
                                         const VertexBufferHandle handle, double* dst);

/* Reductions returning the FP64 accumulator (raw sums for RMS/RMS_EXP). */
AcResult acDeviceReduceScalDouble(const Device device, const Stream stream,
                                  const ReductionType rtype, const VertexBufferHandle handle,
                                  double* result);
AcResult acDeviceReduceVecDouble(const Device device, const Stream stream,
                                 const ReductionType rtype, const VertexBufferHandle a,
                                 const VertexBufferHandle b, const VertexBufferHandle c,
                                 double* result);

/* ---- reduction without device allocation --------------------------------
 * No counterpart in the reference. For callers that cannot call cudaMalloc
 * (a framework that owns all device memory through its own pool, or a loop
 * that must not pay cudaMalloc's implicit synchronisation): reduces the
 * interior of a caller-owned device field and allocates nothing.
 *   cuda_stream  cudaStream_t to launch on (asynchronous; no synchronisation)
 *   field        device pointer, (nx+6)*(ny+6)*(nz+6) AcReal in the reference
 *                index order i + j*mx + k*mx*my
 *   result       device pointer to one double; receives the FP64 accumulator
 *                (RMS and RMS_EXP as raw sums, like acDeviceReduceScal)
 * Scratch lives in a fixed 128 KiB array of the library on each GPU, so
 * meshes with ny*nz > 1,048,576 are rejected (AC_FAILURE), calls that overlap
 * on the GPU race, and the first call on a device looks up the array's device
 * address (make that first call before any stream capture). The address is
 * kept for the life of the process: a device reset (cudaDeviceReset) or a
 * destroyed primary context between calls is not supported. */
AcResult acReduceScalNoAlloc(void* cuda_stream, const ReductionType rtype, const AcReal* field,
                             const int nx, const int ny, const int nz, double* result);

#ifdef __cplusplus
} /* extern "C" */
#endif
