/*
 * acoustic_amr_b200.h — C ABI of the B200 engine's AMR pressure backend.
 *
 * Drop-in for the reference's csrc/include/acoustic_amr.h (implemented there
 * by csrc/kernels/acoustic_amr.cpp): the same 27 amr_* entry points, argument
 * order and meaning, array layouts and return codes, so a rebuilt co-evolver
 * or pressure backend (csrc/kernels/acoustic_pressure_backend.cpp:388-569)
 * links against libacoustic_fdtd_b200.so instead.  The per-step work
 * (velocity gather, plate boundary faces, CSR divergence and pressure update,
 * wall cells, divergence check, Kirchhoff plate) runs on the GPU; create-time
 * coefficients are computed on the host with the reference's arithmetic.
 *
 * Calls are synchronous: each returns after its work (and any read-back) has
 * finished.  A handle is not thread-safe.  Each reference declaration is
 * cited by line in csrc/include/acoustic_amr.h.
 */
#pragma once
#include <stdint.h>

#if defined(__GNUC__)
#define AMR_B200_API __attribute__((visibility("default")))
#else
#define AMR_B200_API
#endif

#ifndef SK_OK
#define SK_OK 0
#define SK_ERR_NULL_STATE -1
#define SK_ERR_DIM_MISMATCH -2
#define SK_ERR_DIVERGED -3
#endif
#define AMR_B200_ERR_CUDA -4   /* engine extension: a CUDA call failed (amr_b200_last_error) */

#ifndef AMR_BORDER_ANECHOIC
#define AMR_BORDER_ANECHOIC 0
#define AMR_BORDER_ROOM_PANEL 1
#define AMR_BORDER_TRANSMISSION 2
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct AcousticAMRState AcousticAMRState;

/* acoustic_amr.h:20-35 */
AMR_B200_API AcousticAMRState* amr_create(int n_cells, const double* cell_centers, const double* cell_volumes,
                                          const double* open_volume_frac, const uint8_t* cell_types,
                                          int n_faces, const int32_t* face_cell_neg,
                                          const int32_t* face_cell_pos, const double* face_area,
                                          const double* face_open_frac, const double* face_distance,
                                          double c, double rho_air, double min_dx, int gradient_order);
/* acoustic_amr.h:44-45 */
AMR_B200_API const char* amr_get_last_create_error_stage(void);
AMR_B200_API const char* amr_get_last_create_error_message(void);
/* acoustic_amr.h:53-55 */
AMR_B200_API int amr_get_create_progress_active(void);
AMR_B200_API int amr_get_create_progress_done_faces(void);
AMR_B200_API int amr_get_create_progress_total_faces(void);
/* acoustic_amr.h:57-60 */
AMR_B200_API void amr_destroy(AcousticAMRState* st);
AMR_B200_API int amr_step(AcousticAMRState* st, int n_steps);
AMR_B200_API int amr_reset(AcousticAMRState* st);
/* acoustic_amr.h:62-65 */
AMR_B200_API int amr_inject_pressure_nearest(AcousticAMRState* st, const double* xyz, float value);
/* acoustic_amr.h:67-70, :78-81, :83-86 */
AMR_B200_API int amr_get_pressure(const AcousticAMRState* st, float* out_pressure, int out_count);
AMR_B200_API int amr_get_cell_centers(const AcousticAMRState* st, float* out_xyz, int n_cells_3);
AMR_B200_API int amr_get_velocity(const AcousticAMRState* st, float* out_velocity, int out_count);
/* acoustic_amr.h:88-89 */
AMR_B200_API double amr_get_dt(const AcousticAMRState* st);
AMR_B200_API int amr_get_step_count(const AcousticAMRState* st);
/* acoustic_amr.h:102-106 */
AMR_B200_API int amr_scatter_pressure_uniform(const AcousticAMRState* st, int Nx, int Ny, int Nz,
                                              const double bmin[3], const double bmax[3], float* out);
/* acoustic_amr.h:132-141 */
AMR_B200_API int amr_set_border_condition(AcousticAMRState* st, int mode, float sigma_order,
                                          float R_reflection, float border_Z_match, int n_pml,
                                          const double* bounds_min, const double* bounds_max);
/* acoustic_amr.h:165-187 */
AMR_B200_API int amr_setup_plate(AcousticAMRState* st, int plate_Nx, int plate_Ny, float plate_dx,
                                 const float plate_origin[3], const uint8_t* plate_active,
                                 float plate_rho_h, float plate_D, float plate_alpha_M, float plate_beta_K,
                                 int n_active_plate, const int32_t* plate_active_flat_idx,
                                 const int32_t* face_above_starts, const int32_t* face_above_idx,
                                 const float* face_above_wgt, const int32_t* face_below_starts,
                                 const int32_t* face_below_idx, const float* face_below_wgt,
                                 const int32_t* cell_above, const int32_t* cell_below);
/* acoustic_amr.h:195-210 */
AMR_B200_API int amr_set_bridge_plate_sources(AcousticAMRState* st, int n, const int32_t* idx, const float* wgt);
AMR_B200_API int amr_set_neck_plate_sources(AcousticAMRState* st, int n, const int32_t* idx, const float* wgt);
/* acoustic_amr.h:226-244 */
AMR_B200_API int amr_inject_bridge_drive(AcousticAMRState* st, const float* cell_drives, int n_cells,
                                         float force_scale);
AMR_B200_API int amr_inject_plate_force(AcousticAMRState* st, int n, const int32_t* plate_idx,
                                        const float* wgt, float total_force_N);
/* acoustic_amr.h:256-283 */
AMR_B200_API int amr_sample_plate_displacement_batch(const AcousticAMRState* st, int n_points, const int* idx4,
                                                     const float* wgt4, float* out_w);
AMR_B200_API int amr_sample_plate_weighted(const AcousticAMRState* st, int n, const int* plate_idx,
                                           const float* wgt, float* out_w);
AMR_B200_API int amr_get_plate_displacement(const AcousticAMRState* st, float* out, int out_len);
/* acoustic_amr.h:301-327 */
AMR_B200_API int amr_setup_mic_samplers(AcousticAMRState* st, int n_mics, const float* pos_xyz,
                                        const float* axis_xyz, int need_velocity);
AMR_B200_API int amr_sample_mics(const AcousticAMRState* st, int n_mics, float* out_p, float* out_vx,
                                 float* out_vy, float* out_vz);

/* ---- engine extensions (no counterpart in the reference) ---- */

/* Last CUDA error or argument problem of an amr_* call (shared by threads). */
AMR_B200_API const char* amr_b200_last_error(void);
/* Kernels launched on the handle so far. */
AMR_B200_API long long amr_b200_launch_count(const AcousticAMRState* st);
/* Queue n_steps steps without waiting (a diverged step is latched on the
 * device and the later steps of the window are skipped there);
 * amr_b200_synchronize waits and returns SK_OK or SK_ERR_DIVERGED, leaving the
 * step count where amr_step would have left it. */
AMR_B200_API int amr_b200_step_async(AcousticAMRState* st, int n_steps);
AMR_B200_API int amr_b200_synchronize(AcousticAMRState* st);
/* CUDA-event timing of the step kernels on the handle's stream: enable, then
 * read the summed kernel time (ms) and the number of timed steps. */
AMR_B200_API int amr_b200_profile(AcousticAMRState* st, int enable);
AMR_B200_API int amr_b200_profile_read(AcousticAMRState* st, double* total_ms, long long* steps);

#ifdef __cplusplus
}
#endif
