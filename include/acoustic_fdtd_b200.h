/*
 * acoustic_fdtd_b200.h — C ABI of the B200 (sm_100a) acoustic FDTD engine.
 *
 * Drop-in for the reference's csrc/include/acoustic_fdtd.h
 * (sangderenard/spectral-analyzer): the 26 fdtd_* entry points below keep the
 * reference's names, signatures, argument meaning, array layouts and return
 * codes, so a caller of that header (the pybind AcousticFDTD wrapper,
 * csrc/bindings/pybind_kernels.cpp:5473-5664, or the uniform co-evolver,
 * csrc/kernels/acoustic_coevolver.cpp:1015-2205) relinks against
 * libacoustic_fdtd_b200.so unchanged.  The fields live in GPU memory; every
 * host array crossing this ABI is caller-owned and copied.
 *
 * Physics and numerics are the reference's: staggered p/Vx/Vy/Vz leapfrog,
 * 4th-order interior gradient and divergence, cubic-graded PML, rigid walls,
 * cut-cell face fractions, Kirchhoff plate.  In float32 the engine rounds
 * exactly like the reference compiled without FMA contraction, so fields,
 * traces and return codes are bit-identical.
 *
 * Layouts seen through this ABI are the reference's (acoustic_fdtd.h:67-71,
 * :430-437): P index k + Nz*(j + Ny*i); Vx k + Nz*(j + Ny*i) for i < Nx-1;
 * Vy k + Nz*(j + (Ny-1)*i); Vz k + (Nz-1)*(j + Ny*i).  On the device every field
 * is stored padded as [Nx][Ny][Sz] with Sz = Nz rounded up to a multiple of 8
 * (fdtd_b200_field_layout).
 *
 * Threading: a handle is not thread-safe (as in the reference).  Calls that
 * return data or a status synchronise the handle's stream before returning;
 * fdtd_step synchronises only when a stability check or the plate guard runs
 * inside the call (every 256 steps, or every step while a plate is active).
 *
 * Codes: FDTD_OK 0, FDTD_ERR_NULL -1, FDTD_ERR_DIM -2, FDTD_ERR_UNSTABLE -3 as
 * in the reference; the engine adds FDTD_ERR_CUDA -4 (CUDA runtime failure;
 * fdtd_b200_last_error has the text) and FDTD_ERR_ARG -5 (invalid argument to
 * an extension, or an out-of-range index that the reference would have read
 * out of bounds).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_B200_API __attribute__((visibility("default")))

#define FDTD_AIR   ((uint8_t)0)
#define FDTD_WALL  ((uint8_t)1)
#define FDTD_PLATE ((uint8_t)2)
#define FDTD_PML   ((uint8_t)3)

#define FDTD_OK            0
#define FDTD_ERR_NULL     (-1)
#define FDTD_ERR_DIM      (-2)
#define FDTD_ERR_UNSTABLE (-3)
#define FDTD_ERR_CUDA     (-4)
#define FDTD_ERR_ARG      (-5)

typedef struct AcousticFDTDState AcousticFDTDState;

/* ===================== reference entry points (acoustic_fdtd.h) ===================== */

/* acoustic_fdtd.h:137-152.  Builds the solver on the current CUDA device and
 * allocates its fields there.  NULL on invalid arguments, when no CUDA device
 * is usable, or when device memory runs out. */
FDTD_B200_API AcousticFDTDState* fdtd_create(
    int Nx, int Ny, int Nz, float dx, float c, float rho_air,
    const uint8_t* cell_type, int plate_iz, const uint8_t* plate_active,
    float plate_mass_density, float plate_stiffness_D,
    float plate_alpha_M, float plate_beta_K, int n_pml);

/* acoustic_fdtd.h:155. */
FDTD_B200_API void fdtd_destroy(AcousticFDTDState* st);

/* acoustic_fdtd.h:171-175.  Weights normalised by the sum of |w|. */
FDTD_B200_API int fdtd_set_bridge_sources(AcousticFDTDState* st, int n_cells,
                                          const int* cell_indices, const float* weights);

/* acoustic_fdtd.h:184-188.  Disabled in the reference; returns FDTD_ERR_UNSTABLE. */
FDTD_B200_API int fdtd_inject_bridge(AcousticFDTDState* st, float signal_val,
                                     float signal_ddt, float force_scale);

/* acoustic_fdtd.h:206-209.  Accumulates into the plate load consumed by the next step. */
FDTD_B200_API int fdtd_inject_bridge_drive(AcousticFDTDState* st, const float* cell_drives,
                                           float force_scale);

/* acoustic_fdtd.h:219-224. */
FDTD_B200_API int fdtd_inject_plate_force(AcousticFDTDState* st, int n_plate,
                                          const int* plate_indices, const float* weights,
                                          float total_force_N);

/* acoustic_fdtd.h:246-250.  NULL leaves a component unchanged. */
FDTD_B200_API int fdtd_set_face_fractions(AcousticFDTDState* st, const float* vx_frac,
                                          const float* vy_frac, const float* vz_frac);

/* acoustic_fdtd.h:255-260. */
FDTD_B200_API int fdtd_sample_plate_weighted(const AcousticFDTDState* st, int n_plate,
                                             const int* plate_indices, const float* weights,
                                             float* out_w);

/* acoustic_fdtd.h:279-284. */
FDTD_B200_API int fdtd_precompute_pressure_samplers(const AcousticFDTDState* st, int n_rec,
                                                    const float* rec_xyz, int* out_idx8,
                                                    float* out_wgt8);

/* acoustic_fdtd.h:294-300. */
FDTD_B200_API int fdtd_precompute_velocity_samplers(const AcousticFDTDState* st, int n_rec,
                                                    const float* rec_xyz,
                                                    int* out_vx_idx8, float* out_vx_wgt8,
                                                    int* out_vy_idx8, float* out_vy_wgt8,
                                                    int* out_vz_idx8, float* out_vz_wgt8);

/* acoustic_fdtd.h:306-311. */
FDTD_B200_API int fdtd_sample_pressure_precomputed(const AcousticFDTDState* st, int n_rec,
                                                   const int* idx8, const float* wgt8,
                                                   float* out_p);

/* acoustic_fdtd.h:317-324. */
FDTD_B200_API int fdtd_sample_velocity_precomputed(const AcousticFDTDState* st, int n_rec,
                                                   const int* vx_idx8, const float* vx_wgt8,
                                                   const int* vy_idx8, const float* vy_wgt8,
                                                   const int* vz_idx8, const float* vz_wgt8,
                                                   float* out_vx, float* out_vy, float* out_vz);

/* acoustic_fdtd.h:338.  Plate update, velocity update, face BCs, pressure
 * update, and the 256-step stability check, n_steps times. */
FDTD_B200_API int fdtd_step(AcousticFDTDState* st, int n_steps);

/* acoustic_fdtd.h:341, :344. */
FDTD_B200_API int fdtd_get_step_count(const AcousticFDTDState* st);
FDTD_B200_API float fdtd_get_dt(const AcousticFDTDState* st);

/* acoustic_fdtd.h:347.  Zeroes P, V and the plate; keeps geometry. */
FDTD_B200_API int fdtd_reset(AcousticFDTDState* st);

/* acoustic_fdtd.h:359-363, :372-376. */
FDTD_B200_API int fdtd_get_pressure_field(const AcousticFDTDState* st, float* out, int out_len);
/* One pressure plane, as acoustic_fdtd_bridge.py:737-757 (get_volume_slice)
 * returns it, without copying the whole field: axis 0 -> (Ny, Nz) at i = idx,
 * 1 -> (Nx, Nz) at j = idx, 2 -> (Nx, Ny) at k = idx; idx < 0 is the mid
 * plane, idx past the end the last plane.  out_len must equal the plane's
 * size (FDTD_ERR_DIM); axis outside 0..2 is FDTD_ERR_ARG. */
FDTD_B200_API int fdtd_b200_get_volume_slice(const AcousticFDTDState* st, int axis, int idx, float* out,
                                             int out_len);
FDTD_B200_API int fdtd_get_plate_displacement(const AcousticFDTDState* st, float* out,
                                              int out_len);

/* acoustic_fdtd.h:396-402. */
FDTD_B200_API int fdtd_sample_plate_displacement_batch(const AcousticFDTDState* st,
                                                       int n_points, const int* saddle_idx4,
                                                       const float* saddle_wgt4, float* out_w);

/* acoustic_fdtd.h:413-418. */
FDTD_B200_API int fdtd_sample_pressure(const AcousticFDTDState* st, int n_rec,
                                       const float* rec_xyz, float* out_p);

/* acoustic_fdtd.h:441-446, :449-458. */
FDTD_B200_API void fdtd_get_velocity_dims(const AcousticFDTDState* st, int* Nvx, int* Nvy,
                                          int* Nvz);
FDTD_B200_API int fdtd_get_velocity_x(const AcousticFDTDState* st, float* out, int out_len);
FDTD_B200_API int fdtd_get_velocity_y(const AcousticFDTDState* st, float* out, int out_len);
FDTD_B200_API int fdtd_get_velocity_z(const AcousticFDTDState* st, float* out, int out_len);

/* acoustic_fdtd.h:476-483. */
FDTD_B200_API int fdtd_sample_velocity(const AcousticFDTDState* st, int n_rec,
                                       const float* rec_xyz, float* out_vx, float* out_vy,
                                       float* out_vz);

/* acoustic_fdtd.h:499-506. */
FDTD_B200_API int fdtd_get_surface_emission(const AcousticFDTDState* st, int n_surf,
                                            const float* surf_xyz, const float* surf_normals,
                                            float* out_P, float* out_vn);

/* ============================ engine extensions ============================ */

/* Device-memory layout of one field: row stride (floats) and bytes per field. */
FDTD_B200_API int fdtd_b200_field_layout(int Nx, int Ny, int Nz, int* row_stride,
                                         size_t* field_bytes);

/* fdtd_create on CUDA device `device` (-1 = current).  When `fields` is
 * non-NULL it holds eight device pointers {P0, P1, Vx0, Vy0, Vz0, Vx1, Vy1,
 * Vz1} (two pressure buffers and two velocity sets), each at least
 * field_bytes long and 16-byte aligned (e.g. torch tensors); the engine uses
 * them instead of allocating, zeroes them, and never frees them. */
FDTD_B200_API AcousticFDTDState* fdtd_b200_create_ex(
    int Nx, int Ny, int Nz, float dx, float c, float rho_air,
    const uint8_t* cell_type, int plate_iz, const uint8_t* plate_active,
    float plate_mass_density, float plate_stiffness_D,
    float plate_alpha_M, float plate_beta_K, int n_pml,
    int device, float* const* fields);

/* Per-face absorption: a6 = {x_lo, x_hi, y_lo, y_hi, z_lo, z_hi}, each > 0,
 * scales the PML's sigma_max on that face.  All ones = the reference. */
FDTD_B200_API int fdtd_b200_set_face_absorption(AcousticFDTDState* st, const float* a6);

/* One pressure deposit with the reference's open-cell rule
 * (acoustic_fdtd.cpp:840-872); returns the number of cells written. */
FDTD_B200_API int fdtd_b200_add_pressure(AcousticFDTDState* st, int cell_index, float amp);

/* Point source: before the step that starts at step count n (0 <= n < n_signal)
 * signal[n] is deposited at cell_index with the open-cell rule.  n_signal = 0
 * removes the source. */
FDTD_B200_API int fdtd_b200_set_point_source(AcousticFDTDState* st, int cell_index,
                                             const float* signal, int n_signal);

/* Receivers: after every step each receiver's 8-tap pressure sample (the
 * layout of fdtd_precompute_pressure_samplers) is appended to a device trace
 * of up to `capacity` steps.  n_rec = 0 removes them. */
FDTD_B200_API int fdtd_b200_set_receivers(AcousticFDTDState* st, int n_rec, const int* idx8,
                                          const float* wgt8, int capacity);

/* Copies the recorded traces, [n_recorded][n_rec] float32, and clears them. */
FDTD_B200_API int fdtd_b200_get_traces(AcousticFDTDState* st, float* out, int out_len,
                                       int* n_recorded);

/* Stream the handle works on (a cudaStream_t; NULL = the handle's own stream). */
FDTD_B200_API int fdtd_b200_set_stream(AcousticFDTDState* st, void* stream);
FDTD_B200_API void* fdtd_b200_get_stream(const AcousticFDTDState* st);

/* Launches n_steps without waiting and without stopping at a failed stability
 * check; the first failure is latched and reported by fdtd_b200_synchronize. */
FDTD_B200_API int fdtd_b200_step_async(AcousticFDTDState* st, int n_steps);

/* Waits for the handle's stream; returns FDTD_OK, FDTD_ERR_UNSTABLE (latched
 * by an async step) or FDTD_ERR_CUDA.  Clears the latch. */
FDTD_B200_API int fdtd_b200_synchronize(AcousticFDTDState* st);

/* Step-kernel selection: 0 automatic (fused single pass for open rooms and
 * for walled scenes of at least 2^22 cells, two-pass for smaller walled
 * scenes), 1 two-pass, 2 fused.  Walled scenes (solid cells, face fractions,
 * an active plate) run the single pass with the walled rules; both kernels
 * give the same results bit for bit.  FDTD_ERR_ARG for 2 when the row
 * padding does not allow the single pass. */
FDTD_B200_API int fdtd_b200_set_kernel(AcousticFDTDState* st, int mode);
FDTD_B200_API int fdtd_b200_get_kernel(const AcousticFDTDState* st);

/* Failure-path hook for tests of the fused step's bounded waits (no reference
 * counterpart).  From the next fused step on, the TMA load of pressure plane
 * `plane` (0 .. Nx-1) is armed on its mbarrier but never issued, so every CTA
 * that needs it gives up after `wait_us` microseconds (0: the normal bound of
 * 2 s), records a timeout status and exits, leaving that step incomplete.
 * fdtd_b200_synchronize then returns FDTD_ERR_CUDA ("load wait timed out")
 * until fdtd_reset; the CUDA context stays usable.  plane -1 turns it off. */
FDTD_B200_API int fdtd_b200_debug_hold_load(AcousticFDTDState* st, int plane, int wait_us);

/* Device pointers of the current fields: out5 = {P (current), P (next), Vx, Vy, Vz}. */
FDTD_B200_API int fdtd_b200_device_fields(const AcousticFDTDState* st, void** out5);

/* Progress of a room: its step count, the rotating phase of the 256-step
 * stability check, and the step whose source sample is already in P (-1:
 * none; a batch deposits the next step's sample ahead of it).  With the
 * current fields (fdtd_b200_device_fields) they are the state a later step
 * depends on: copying the fields into another handle of the same room and
 * setting its progress resumes the room exactly (a serving pre-emption
 * snapshot). */
FDTD_B200_API int fdtd_b200_get_progress(const AcousticFDTDState* st, int* step_count, int* check_phase,
                                         int* deposited_step);
FDTD_B200_API int fdtd_b200_set_progress(AcousticFDTDState* st, int step_count, int check_phase,
                                         int deposited_step);

/* CUDA-event timing of the main step kernel(s) on the handle's stream. */
FDTD_B200_API int fdtd_b200_profile(AcousticFDTDState* st, int enable);
FDTD_B200_API int fdtd_b200_profile_read(AcousticFDTDState* st, double* total_ms,
                                         long long* launches, long long* kernel_launches);

/* No counterpart in the reference.  fdtd_sample_pressure_precomputed for
 * callers that cannot allocate — e.g. a real-time audio callback sampling the
 * microphones, where a cudaMalloc or cudaMallocHost may block on driver locks
 * for an unbounded time.  It never calls cudaMalloc/cudaFree or any
 * allocating routine: its index/weight inputs and its results are staged in
 * one fixed device array (272 KB, shared by all handles on a device and kept
 * until the process exits).  At most 4096 receivers per call (FDTD_ERR_ARG
 * beyond, with the reason in fdtd_b200_last_error).  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and
 * keeps it for the life of the process; make that first call before any CUDA
 * stream capture starts, and do not use this function after a
 * cudaDeviceReset of that device in the same process (the kept address is
 * then stale).  The call copies from and to pageable host memory on the
 * handle's stream and ends with a synchronisation of that stream: it blocks
 * until every step already queued on the handle has finished, so a real-time
 * caller should call it only when no steps are queued, and it must not be
 * made while the handle's stream is being captured.  Each call overwrites
 * what it uses of the array, so nothing in it has to start at zero, but calls
 * that overlap on the GPU (other threads or streams) race on it.  Same
 * arguments, index checks and results as fdtd_sample_pressure_precomputed. */
FDTD_B200_API int fdtd_b200_sample_pressure_noalloc(const AcousticFDTDState* st, int n_rec,
                                                   const int* idx8, const float* wgt8,
                                                   float* out_p);

/* ---- batched stepping of independent rooms (serving) ----
 * A batch advances several solver handles together: each batched step is one
 * persistent kernel over the work items (tile x plane segment) of every member
 * below its step limit, plus one epilogue kernel (receivers, step counters,
 * 256-step check, next source sample).  Members must be open rooms (no walls,
 * fractions or active plate).  A member's arithmetic is the same as in
 * fdtd_step, so its fields and traces are bit-identical alone and in a batch.
 * Do not call other functions on a member while the batch holds it: take it
 * out with fdtd_b200_batch_set (which first writes every member's progress
 * back to its handle) or read its progress with fdtd_b200_batch_sync. */
typedef struct FdtdB200Batch FdtdB200Batch;
FDTD_B200_API FdtdB200Batch* fdtd_b200_batch_create(int device);
FDTD_B200_API void fdtd_b200_batch_destroy(FdtdB200Batch* b);
/* Replace the members; member q advances until its step count reaches limits[q]. */
FDTD_B200_API int fdtd_b200_batch_set(FdtdB200Batch* b, AcousticFDTDState* const* members,
                                      const int* limits, int n);
/* Work-item tile: tile_k = 128 (8 rows x 128 columns, the default) or 64
 * (16 rows x 64 columns, less idle width for rooms with small Nz); takes
 * effect at the next batch_set. */
FDTD_B200_API int fdtd_b200_batch_set_tile(FdtdB200Batch* b, int tile_k);
/* Planes per work item (0 = automatic); takes effect at the next batch_set. */
FDTD_B200_API int fdtd_b200_batch_set_segment(FdtdB200Batch* b, int planes);
/* Launch n_steps batched steps without waiting; use_graph = 1 captures them
 * once as a CUDA graph per n_steps and replays it (the graph stays valid
 * across member sets; it is re-captured only when a set outgrows the
 * descriptor capacity). */
FDTD_B200_API int fdtd_b200_batch_step(FdtdB200Batch* b, int n_steps, int use_graph);
/* Wait, then write each member's step count, buffers and traces back to its
 * handle; steps_out[q] = step count, status_out[q] = 0 or FDTD_ERR_UNSTABLE
 * (a failed 256-step check, latched; the member kept stepping). */
FDTD_B200_API int fdtd_b200_batch_sync(FdtdB200Batch* b, int* steps_out, int* status_out);
FDTD_B200_API long long fdtd_b200_batch_launch_count(const FdtdB200Batch* b);

/* ---- storage-precision study (no reference counterpart) ----
 * An open room (no walls, fractions or plate; PML with per-face scales a6,
 * NULL = all 1) stepped by the two-pass update with the fields stored as
 *   mode 0 FP32, 1 FP64 (arithmetic in double: the GPU oracle),
 *   2 BF16, 3 FP16, 4 BF16 + BF16 residual, 5 FP16 + FP16 residual;
 * modes 2-5 compute in FP32 and round each stored value; the residual modes
 * keep the FP32-formed remainder x - rn16(x) beside it (loads return the sum).
 * FP16 fields are stored times p_scale (P) or v_scale (V), powers of two
 * (<= 0 picks 2^10 and 2^19, right for source samples of order 1).
 * Sources are deposited before a step, receivers (8 taps, summed in double)
 * record after it, as fdtd_step + fdtd_sample_pressure_precomputed do.
 * The 16-bit modes (2-5) step by default with a single-pass kernel that
 * reads and writes each stored field once (fdtd_b200_prec_set_kernel); it
 * produces the two-pass update's stored bits, and steps that take an energy
 * audit run the two-pass update. */
typedef struct FdtdB200Prec FdtdB200Prec;
FDTD_B200_API FdtdB200Prec* fdtd_b200_prec_create(int Nx, int Ny, int Nz, double dx, double c,
                                                  double rho_air, int n_pml, const float* a6,
                                                  int mode, float p_scale, float v_scale,
                                                  int device);
FDTD_B200_API void fdtd_b200_prec_destroy(FdtdB200Prec* p);
FDTD_B200_API double fdtd_b200_prec_dt(const FdtdB200Prec* p);
/* Source cell (flat reference index) and its per-step samples. */
FDTD_B200_API int fdtd_b200_prec_set_source(FdtdB200Prec* p, int cell, const double* signal,
                                            int n);
/* Receivers as 8-tap samplers (fdtd_precompute_pressure_samplers layout),
 * trace capacity in steps, and capacity of the energy-audit log. */
FDTD_B200_API int fdtd_b200_prec_set_receivers(FdtdB200Prec* p, int n_rec, const int* idx8,
                                               const double* wgt8, int capacity,
                                               int audit_capacity);
/* Launch n_steps steps; with audit_every > 0 the velocity pass of every step
 * whose index is a multiple of it also sums the discrete energy in double. */
FDTD_B200_API int fdtd_b200_prec_step(FdtdB200Prec* p, int n_steps, int audit_every);
FDTD_B200_API int fdtd_b200_prec_get_traces(FdtdB200Prec* p, double* out, int out_len,
                                            int* n_recorded);
/* Rows (step n, potential part sum p^2/(rho c^2), energy E^n) with
 * E^n = dx^3/2 (sum (p^n)^2/(rho c^2) + rho sum v^{n-1/2} v^{n+1/2}). */
FDTD_B200_API int fdtd_b200_prec_get_energy(FdtdB200Prec* p, double* out3, int out_rows,
                                            int* n_out);
/* Current pressure, reference cell order, widened to double. */
FDTD_B200_API int fdtd_b200_prec_get_pressure(FdtdB200Prec* p, double* out, int out_len);
/* Step kernel of a 16-bit mode: 1 single pass (the default), 0 two-pass.
 * FDTD_ERR_ARG for 1 in the FP32 / FP64 modes. */
FDTD_B200_API int fdtd_b200_prec_set_kernel(FdtdB200Prec* p, int kernel);
FDTD_B200_API int fdtd_b200_prec_get_kernel(const FdtdB200Prec* p);
/* Kernels launched by fdtd_b200_prec_step since create. */
FDTD_B200_API long long fdtd_b200_prec_launch_count(const FdtdB200Prec* p);
/* The handle's CUDA stream (cudaStream_t), for events around its steps. */
FDTD_B200_API void* fdtd_b200_prec_stream(const FdtdB200Prec* p);

/* ---- gradient w.r.t. per-cell absorption (no reference counterpart) ----
 * An open room whose absorption is a per-cell field a_c = alpha_c * dt in
 * [0, 1] (the reference stores alpha per cell, acoustic_fdtd.cpp:64; here the
 * whole field is an input): P damping 1/(1 + a_c), face damping
 * 1 - (a_L + a_R)/2.  fdtd_b200_adj_forward runs n steps from rest (source
 * deposited before each step, receivers recorded after it) and, with
 * keep_checkpoints, stores p^n and v^{n-1/2} every checkpoint_every steps;
 * fdtd_b200_adj_backward takes dL/dy (per step and receiver, the layout of
 * the traces) and returns dL/da in reference cell order, recomputing the
 * forward segment by segment and running the adjoint kernels backwards.
 * use_double = 1 computes everything in double (for finite-difference checks);
 * otherwise the arithmetic is float and the gradient accumulates in double.
 * a_cell and grad_out may be host or device pointers. */
typedef struct FdtdB200Adj FdtdB200Adj;
FDTD_B200_API FdtdB200Adj* fdtd_b200_adj_create(int Nx, int Ny, int Nz, double dx, double c,
                                                double rho_air, int use_double,
                                                int checkpoint_every, int device);
FDTD_B200_API void fdtd_b200_adj_destroy(FdtdB200Adj* h);
FDTD_B200_API double fdtd_b200_adj_dt(const FdtdB200Adj* h);
FDTD_B200_API long long fdtd_b200_adj_launch_count(const FdtdB200Adj* h);
/* a_cell: Nx*Ny*Nz values of value_bytes (4 = float, 8 = double). */
FDTD_B200_API int fdtd_b200_adj_set_absorption(FdtdB200Adj* h, const void* a_cell, int len,
                                               int value_bytes);
FDTD_B200_API int fdtd_b200_adj_set_source(FdtdB200Adj* h, int cell, const double* signal, int n);
/* Receivers as 8-tap samplers; max_steps bounds the forward length. */
FDTD_B200_API int fdtd_b200_adj_set_receivers(FdtdB200Adj* h, int n_rec, const int* idx8,
                                              const double* wgt8, int max_steps);
/* traces_out (host, may be NULL): n_steps x n_rec, widened to double. */
FDTD_B200_API int fdtd_b200_adj_forward(FdtdB200Adj* h, int n_steps, int keep_checkpoints,
                                        double* traces_out);
/* dloss_dtrace (host): n_steps x n_rec of the last checkpointed forward;
 * grad_out: Nx*Ny*Nz doubles. */
FDTD_B200_API int fdtd_b200_adj_backward(FdtdB200Adj* h, const double* dloss_dtrace,
                                         double* grad_out);

/* ---- one slab of a room split along i across GPUs (no reference counterpart) ----
 * The slab owns global planes [i0, i1) (at least 3) of an open room and keeps
 * three ghost planes each side: local plane l = global plane i0 - 3 + l,
 * *local_planes = i1 - i0 + 6 planes of [Ny][Sz] floats per field.  The
 * caller allocates eight zeroed fields {P0, P1, Vx0, Vy0, Vz0, Vx1, Vy1, Vz1}
 * of that size (two pressure buffers, two velocity sets) and exchanges ghost
 * planes with the neighbours: P of the current buffer (fdtd_b200_slab_current)
 * planes 3,4,5 to the left neighbour's own+3 .. own+5 and own .. own+2 to the
 * right neighbour's 0 .. 2; Vx of the current set (fdtd_b200_slab_vset)
 * planes 3,4 to the left neighbour's own+3, own+4 and own+1, own+2 to the
 * right neighbour's 1, 2.
 * Fused step: deposit(n), step, exchange P and Vx, record.
 * Two-pass step: deposit(n), velocity, exchange Vx, pressure, exchange P, record.
 * The source and receiver taps may lie in ghost planes (a source there is
 * deposited into the ghost copy too); set them on every slab whose planes
 * (ghosts included) hold them.  Kernels run on the stream of
 * fdtd_b200_slab_set_stream (0 = the legacy default stream). */
typedef struct FdtdB200Slab FdtdB200Slab;
FDTD_B200_API int fdtd_b200_slab_layout(int Nx, int Ny, int Nz, int i0, int i1, int* local_planes,
                                        int* sz);
FDTD_B200_API FdtdB200Slab* fdtd_b200_slab_create(int Nx, int Ny, int Nz, int i0, int i1, float dx,
                                                  float c, float rho_air, int n_pml,
                                                  const float* a6, float* const* fields,
                                                  int device);
FDTD_B200_API void fdtd_b200_slab_destroy(FdtdB200Slab* h);
FDTD_B200_API int fdtd_b200_slab_set_stream(FdtdB200Slab* h, void* stream);
FDTD_B200_API float fdtd_b200_slab_dt(const FdtdB200Slab* h);
/* Index (0 or 1) of the field holding the current pressure / velocity set. */
FDTD_B200_API int fdtd_b200_slab_current(const FdtdB200Slab* h);
FDTD_B200_API int fdtd_b200_slab_vset(const FdtdB200Slab* h);
FDTD_B200_API long long fdtd_b200_slab_launch_count(const FdtdB200Slab* h);
/* cell: global flat index; ignored (no source here) when outside this slab's planes. */
FDTD_B200_API int fdtd_b200_slab_set_source(FdtdB200Slab* h, int cell, const float* signal, int n);
/* Receivers as 8-tap samplers in global flat indices, every tap inside this slab's planes. */
FDTD_B200_API int fdtd_b200_slab_set_receivers(FdtdB200Slab* h, int n_rec, const int* idx8,
                                               const float* wgt8, int capacity);
FDTD_B200_API int fdtd_b200_slab_deposit(FdtdB200Slab* h, int n);
/* Deposit amp (from the host) into this slab's copy of a cell, global flat
 * index; a no-op when the slab holds no copy of the cell. */
FDTD_B200_API int fdtd_b200_slab_add_pressure(FdtdB200Slab* h, int cell, float amp);
/* Read back the receiver samples of the last recorded step (n = the slab's
 * receiver count); waits for the slab's stream. */
FDTD_B200_API int fdtd_b200_slab_read_last(FdtdB200Slab* h, float* out, int n);
/* Fused single-pass step of the own planes (flips both current indices). */
FDTD_B200_API int fdtd_b200_slab_step(FdtdB200Slab* h);
/* The same step in two parts, so that the ghost exchange overlaps the
 * interior: part 1 = the first and last three own planes (what the
 * neighbours keep as ghosts), part 2 = the planes between them, then the
 * buffer flip.  Bit-identical to fdtd_b200_slab_step; part 2 may be launched
 * on another stream (fdtd_b200_slab_set_stream) while part 1's planes are
 * sent. */
FDTD_B200_API int fdtd_b200_slab_step_part(FdtdB200Slab* h, int part);
/* The fused step can also write the neighbours' ghost planes itself (3 planes
 * of the new P, 2 of the new Vx per side), so that only a barrier separates
 * the steps: side 0 = left, 1 = right; fields = the neighbour's eight fields
 * in the same order as fdtd_b200_slab_create's, as pointers writable here
 * (same device, peer access or an IPC mapping), NULL to clear; [peer_i0,
 * peer_i1) = its planes.  Neighbours must step in lockstep. */
FDTD_B200_API int fdtd_b200_slab_set_peer(FdtdB200Slab* h, int side, float* const* fields, int peer_i0,
                                          int peer_i1);
FDTD_B200_API int fdtd_b200_slab_velocity(FdtdB200Slab* h);
FDTD_B200_API int fdtd_b200_slab_pressure(FdtdB200Slab* h);
FDTD_B200_API int fdtd_b200_slab_record(FdtdB200Slab* h);
/* Stability sample of the own cells (global flat phase + 1013 t); *bad = the
 * smallest failing flat index or -1.  Synchronises the stream. */
FDTD_B200_API int fdtd_b200_slab_check(FdtdB200Slab* h, int phase, long long* bad);
FDTD_B200_API int fdtd_b200_slab_get_traces(FdtdB200Slab* h, float* out, int out_len, int* n_rows);

/* One substep of the reference's uniform co-evolver in one call (no reference
 * counterpart): fdtd_inject_bridge_drive(st, cell_drives, drive_scale) when
 * cell_drives is not NULL, fdtd_inject_plate_force(st, n_force, force_idx,
 * force_wgt, force_total_N) when n_force > 0, fdtd_step(st, 1) and
 * fdtd_sample_plate_displacement_batch(st, n_saddle, ...), with the same
 * results and return codes as that sequence (the saddle indices are checked
 * before stepping) and one stream synchronisation instead of two: the plate
 * guard of the step is evaluated on the device and read back together with
 * the saddle samples.  out_saddle_w is written only when the step succeeds.
 * When the handle records no receivers on the device and the step takes no
 * stability check, the device work is replayed from a cached CUDA graph
 * (kept per set of buffers and flags, at most 12 per handle) on the handle's
 * stream; on a stream that cannot be captured it is issued directly. */
FDTD_B200_API int fdtd_b200_substep(AcousticFDTDState* st, const float* cell_drives,
                                    float drive_scale, int n_force, const int* force_idx,
                                    const float* force_wgt, float force_total_N, int n_saddle,
                                    const int* saddle_idx4, const float* saddle_wgt4,
                                    float* out_saddle_w);

/* Number of kernels this handle has launched since creation. */
FDTD_B200_API long long fdtd_b200_launch_count(const AcousticFDTDState* st);

/* Text of the last CUDA error seen by any handle in this process. */
FDTD_B200_API const char* fdtd_b200_last_error(void);

#ifdef __cplusplus
}
#endif
