/*
 * xfdtd_host.h -- C entry points of the C++20 host library (libxfdtd_host.so)
 * for callers that cannot use the C++ API (Python ctypes, test harnesses).
 *
 * A scene file is the line format written by xfdtd_core_b200.scene.Scene:
 * each line becomes the xfdtd:: API call a reference user program would make
 * (Simulation ctor, addObject, addBoundary(PML), addWaveformSource(TFSF3D),
 * CurrentSource, MovieMonitor, NFFFTFrequencyDomain).  These calls have no
 * counterpart in the reference, whose only user interface is C++.
 */
#ifndef XFDTD_HOST_H_
#define XFDTD_HOST_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct xfd_engine;
typedef struct xfdtd_scene xfdtd_scene;

/* Parses `path`, builds the Simulation and runs its set-up (grid, classes,
 * CPML, TFSF, ADE, NF2FF, engine upload) for the scene's step count.
 * precision: 0 = FP64, 1 = FP32, optionally or-ed with XFDTD_SCENE_NO_ENGINE
 * (host set-up only, no GPU needed; only xfdtd_scene_info and
 * xfdtd_scene_coefficients are then usable).  Returns 0 on success. */
#define XFDTD_SCENE_NO_ENGINE 0x100
int xfdtd_scene_open(const char* path, int32_t precision, xfdtd_scene** out);
void xfdtd_scene_close(xfdtd_scene* s);
/* Message of the last failure on this thread. */
const char* xfdtd_host_last_error(void);

/* The engine the scene drives (owned by the scene). */
struct xfd_engine* xfdtd_scene_engine(xfdtd_scene* s);
/* Engine option (xfd_set_option names), applied when the engine is created
 * by the first advance, or at once afterwards (Simulation::setEngineOption). */
int xfdtd_scene_set_engine_option(xfdtd_scene* s, const char* name, int64_t value);
/* Grid size (cells), time step and scene step count. */
int xfdtd_scene_info(xfdtd_scene* s, int32_t n[3], double* dt, int64_t* steps);
/* Queues n time steps (Simulation::advance). */
int xfdtd_scene_advance(xfdtd_scene* s, int64_t n);
/* Waits and copies fields, movie frames and NF2FF currents to the host
 * (Simulation::finish). */
int xfdtd_scene_finish(xfdtd_scene* s);
/* The 18 coefficient arrays in reference shapes (see
 * Simulation::coefficientArrays); each out[q] must hold the array. */
int xfdtd_scene_coefficients(xfdtd_scene* s, double* const out[18]);
/* The TFSF3D set-up (1-D incident grid for every step and the projections);
 * aux = 0 when the scene has no TFSF.  Any output pointer may be NULL;
 * e_inc holds steps*aux, h_inc steps*(aux-1), p_int[a] box_size[a]+1 and
 * p_half[a] box_size[a]+2 doubles. */
int xfdtd_scene_tfsf(xfdtd_scene* s, double* e_inc, double* h_inc, double* const p_int[3],
                     double* const p_half[3], int32_t* aux);
/* Host copy of field `comp` (0..5) after finish, reference shape. */
int xfdtd_scene_field(xfdtd_scene* s, int32_t comp, double* out);
/* Frames of movie `index` (scene order): n_frames and the box shape; with
 * out != NULL copies n_frames*prod(shape) doubles. */
int xfdtd_scene_movie(xfdtd_scene* s, int32_t index, double* out, int64_t capacity,
                      int64_t* n_frames, int32_t shape[3]);
/* Field time monitor `index` (scene order): count = number of steps; with
 * out != NULL writes the time axis then the samples (2*count doubles), like
 * TimeMonitor::output's [time; data] (src/monitor/time_monitor.cpp:11-21). */
int xfdtd_scene_field_time(xfdtd_scene* s, int32_t index, double* out, int64_t capacity,
                           int64_t* count);
/* NF2FF surface currents (complex interleaved, [f][face][ja jb ma mb][nodes]). */
int xfdtd_scene_nf2ff(xfdtd_scene* s, double* out, int64_t capacity, int64_t* count);
/* NF2FF far-field potentials on the GPU (NFFFTFrequencyDomain::farField):
 * complex interleaved [freq][a_theta f_phi a_phi f_theta][angle] for the
 * angles theta x phi (n_theta or n_phi must be 1).  With `sub_dir` non-NULL
 * it also writes them like processFarField, under <dir>/<sub_dir>. */
int xfdtd_scene_far_field(xfdtd_scene* s, int32_t n_theta, const double* theta, int32_t n_phi,
                          const double* phi, const double origin[3], double* out,
                          int64_t capacity, int64_t* count, const char* dir,
                          const char* sub_dir);
/* Writes <dir>/fields/{EX..HZ}.npy, <dir>/<movie>/<step:05d>.npy and
 * <dir>/nf2ff.npy like the reference's Monitor::output (src/monitor/monitor.cpp:42-54). */
/* J = sum_p |F_p|^2 over the E component `field` at the nodes of [box_s,
 * box_e), F_p = dt sum_n E^n(p) exp(-i 2 pi freq n dt), over the next n_steps
 * steps (the scene advances).  With `grad` (capacity >= voxel count), also
 * dJ/deps_r of every voxel of the scene's VoxelObject number `voxel_object`
 * (C order) by the discrete adjoint, saving the state every
 * checkpoint_interval steps.  Returns 0 on success. */
int xfdtd_scene_dft_objective(xfdtd_scene* s, int64_t n_steps, int32_t field,
                              const int32_t box_s[3], const int32_t box_e[3], double freq,
                              int32_t voxel_object, int32_t checkpoint_interval, double* value,
                              double* grad, int64_t capacity);

/* S-parameter S[key] (key = 10 j + i: port j's outgoing wave over source
 * port i's incident wave) of the finished scene's network, one complex value
 * per network frequency as (re, im) pairs; count = 2 n_freqs.
 * Replaces: Network::output (src/network/network.cpp:47-84) without the
 * files; xfdtd_scene_write_outputs writes them under network/. */
int xfdtd_scene_s_parameter(xfdtd_scene* s, int32_t key, double* out, int64_t capacity,
                            int64_t* count);

/* Voltage (kind 0) or current (kind 1) monitor number `index` of the
 * finished scene: [time; data], 2 x n_steps doubles, count = 2 n_steps. */
int xfdtd_scene_line_monitor(xfdtd_scene* s, int32_t kind, int32_t index, double* out,
                             int64_t capacity, int64_t* count);

/* Time-domain NF2FF of the finished scene: 4 x n_bins doubles, w_theta,
 * w_phi, u_theta, u_phi (NFFFTTimeDomain::processFarField).  count = 4 n_bins. */
int xfdtd_scene_nf2ff_td(xfdtd_scene* s, double* out, int64_t capacity, int64_t* count);

int xfdtd_scene_write_outputs(xfdtd_scene* s, const char* dir);

#ifdef __cplusplus
}
#endif

#endif /* XFDTD_HOST_H_ */
