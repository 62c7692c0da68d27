/*
 * xfd_engine.h -- C ABI of the B200 FDTD engine (libxfd_engine.so).
 *
 * The engine owns every device buffer of one 3-D FDTD simulation and runs its
 * time loop on one GPU.  Host code (the C++20 xfdtd::Simulation library, or
 * any FFI) computes the FP64 set-up data -- material classes, curl factors,
 * CPML grading, TFSF incident tables, ADE and lumped coefficients, NF2FF
 * phasors -- and hands it over through these calls.  Host pointers are only
 * borrowed for the duration of a call.  No call throws; each returns an
 * xfd_status and xfd_last_error() describes the most recent failure.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the EMinsight/XFDTD_CORE source tree).  The reference has no C ABI: its
 * hot path is a set of virtual C++ interfaces driven by Domain::run
 * (src/domain/domain.cpp:82-135).
 *
 * Lattice layout.  Every field component, the per-lattice material-class
 * index and the CPML auxiliaries live on the (nx+1) x (ny+1) x (nz+1) node
 * lattice, k fastest.  Component arrays keep the reference shapes
 * (Ex(nx,ny+1,nz+1) ... Hz(nx,ny,nz+1), src/simulation/simulation.cpp:514-528)
 * at the host boundary; the device pads rows to a 32-element pitch.
 *
 * Component order everywhere: 0=Ex 1=Ey 2=Ez 3=Hx 4=Hy 5=Hz; axes 0=x 1=y 2=z;
 * the tangential axes of axis c are a=(c+1)%3 and b=(c+2)%3.
 */
#ifndef XFD_ENGINE_H_
#define XFD_ENGINE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xfd_engine xfd_engine;

typedef enum {
  XFD_OK = 0,
  XFD_ERR_INVALID_ARGUMENT = 1,
  XFD_ERR_CUDA = 2,
  XFD_ERR_UNSUPPORTED = 3,
  XFD_ERR_STATE = 4,
  XFD_ERR_OUT_OF_MEMORY = 5,
  XFD_ERR_NUMERIC = 6,
  XFD_ERR_TIMEOUT = 7  /* a bounded device-side wait ran out of time */
} xfd_status;

typedef enum { XFD_FP64 = 0, XFD_FP32 = 1 } xfd_precision;

typedef struct {
  int32_t nx, ny, nz;   /* cells, CPML included */
  int32_t precision;    /* xfd_precision of fields, coefficients, CPML and ADE state */
  int64_t n_steps;      /* steps of the run: sizes the per-step source tables */
  double dt;
  int32_t device;       /* CUDA device ordinal */
} xfd_grid_desc;

/* Creates an engine with zeroed fields and no boundaries or sources.
 * Replaces: Simulation::init's EMF/coefficient allocation
 * (src/simulation/simulation.cpp:319-371, :514-528). */
xfd_status xfd_create(const xfd_grid_desc* grid, xfd_engine** out);

/* Frees every device and pinned buffer of the engine. */
void xfd_destroy(xfd_engine* e);

/* Message of the last failed call on `e` (or of the last failed xfd_create
 * when e is NULL).  Valid until the next call on the same engine. */
const char* xfd_last_error(const xfd_engine* e);

/* Material classes.  `table` holds n_classes rows of 12 doubles: (ca, cb) for
 * Ex, Ey, Ez, Hx, Hy, Hz, where the E update of component c is
 *   E_c = ca*E_c + cb*( fe_a[x_a]*(H_b - H_b[x_a-1]) - fe_b[x_b]*(H_a - H_a[x_b-1]) )
 * and the H update
 *   H_c = ca*H_c + cb*( fh_b[x_b]*(E_a[x_b+1] - E_a) - fh_a[x_a]*(E_b[x_a+1] - E_b) )
 * with the per-axis curl factors of xfd_set_curl_factors.  `lattice_class`
 * gives the class of every lattice node ((nx+1)*(ny+1)*(nz+1), k fastest).
 * Replaces: the 18 full-grid FDTDUpdateCoefficient arrays
 * (include/xfdtd/calculation_param/fdtd_update_coefficient.h:102-121) filled by
 * CalculationParam::calculateCoefficient (src/calculation_param/calculation_param.cpp:170-264). */
xfd_status xfd_set_material_classes(xfd_engine* e, const double* table, int32_t n_classes,
                                    const uint16_t* lattice_class);

/* Per-node E coefficient overrides: the E update of component comp[q] at
 * node (node[3q], node[3q+1], node[3q+2]) uses (ca[q], cb[q]) instead of its
 * class's pair -- for nodes whose coefficients are all distinct (a block of
 * per-voxel permittivities would otherwise need one class per node).  Only
 * for nodes in the main update range outside CPML layers; call after
 * xfd_set_material_classes, once.  The sweep applies the class pair (ca0,
 * cb0) and a fix-up completes the node: E' = (cb/cb0) E_sweep +
 * (ca - (cb/cb0) ca0) E_old.
 * Replaces: the per-cell coefficients that an Object overriding
 * correctMaterialSpace (include/xfdtd/object/object.h:47) writes into the
 * full-grid coefficient arrays. */
xfd_status xfd_set_e_overrides(xfd_engine* e, int64_t n, const int32_t* node, const int32_t* comp,
                               const double* ca, const double* cb);

/* Halo copy between two engines of one slab decomposition (along x):
 * copies plane `src_plane` of the components comps[0 .. n_comp) (0..5: Ex Ey
 * Ez Hx Hy Hz) of `src`'s current fields into plane `dst_plane` of `dst`'s
 * current fields.  The engines must share the y-z lattice (ny, nz) and the
 * precision; they may sit on different devices (a peer copy, through NVLink
 * where the devices are peers).  Ordering is on the streams: the copy waits
 * for every step queued on `src`, and `src`'s next queued work waits for the
 * copy; `dst`'s next step comes after it on `dst`'s stream.  Asynchronous;
 * xfd_sync(dst) waits for it.
 * Replaces: the reference's per-step MPI halo exchange
 * (MpiSupport::sendRecvHyXHead/Tail etc., src/parallel/mpi_support.cpp:98-229,
 * called from Domain::exchangeH, src/domain/domain.cpp:237-279); this
 * library's slabs exchange the tangential E of one plane instead (the dual
 * scheme, see xfdtd_core_b200/slab.py). */
xfd_status xfd_halo_copy(xfd_engine* dst, int32_t dst_plane, xfd_engine* src, int32_t src_plane,
                         int32_t n_comp, const int32_t* comps);

/* The same planes between an engine and a buffer, for slabs run by one
 * process per GPU (xfdtd_core_b200/slab.py: SlabRank, which moves the buffers
 * between the processes with torch.distributed -- NCCL on device buffers, or
 * gloo on host buffers).  Plane `plane` of each of the n_comp components
 * `comps` (0..5 = Ex Ey Ez Hx Hy Hz) of the engine's current fields, NY x KP
 * values each in the engine's padded layout (xfd_plane_values), from the
 * engine into `buf` (into_engine = 0) or from `buf` into the engine (1),
 * component after component.  `buf` may be device memory of any device or
 * host memory (pinned for speed).  Asynchronous, ordered on the engine's
 * stream after its queued steps; xfd_sync(e) waits for it.
 * Replaces: the buffer side of the reference's halo exchange
 * (MpiSupport::sendRecvHyXHead/Tail, src/parallel/mpi_support.cpp:98-229). */
xfd_status xfd_plane_copy(xfd_engine* e, int32_t plane, int32_t n_comp, const int32_t* comps,
                          void* buf, int32_t into_engine);
/* Values of one padded x-plane of one component: NY x KP. */
int64_t xfd_plane_values(const xfd_engine* e);

/* Per-node H curl-term corrections: after the H sweep of every step, the H
 * component comp[q] at node (node[3q], node[3q+1], node[3q+2]) gets
 *   delta_a[q] * (E_a[x_b+1] - E_a) + delta_b[q] * (E_b[x_a+1] - E_b)
 * added (a = comp+1, b = comp+2 mod 3; the E of the same step) -- for
 * coefficients that scale one curl term of a node but not the other, which
 * the class table's single cb per component cannot hold.  Nodes in the main H
 * range (x < n on every axis), one entry per (node, component); call once.
 * The correction runs between the H and E phases of a split sweep: an engine
 * on a fused sweep moves to the split one (kernel 4 from 7, else 0), and
 * the fused kernels (1, 2, 5, 6, 7) are refused afterwards.  Not batched, no
 * adjoint.
 * Replaces: ThinWire::correctUpdateCoefficient's scaling of chxey, chyex,
 * chzex, chzey next to the wire (src/object/thin_wire.cpp:42-133) in the
 * full-grid coefficient arrays. */
xfd_status xfd_set_h_term_overrides(xfd_engine* e, int64_t n, const int32_t* node,
                                    const int32_t* comp, const double* delta_a,
                                    const double* delta_b);

/* Per-axis curl factors.  fe[a] has n_a+1 entries, 1/(h_size * kappa_e);
 * fh[a] has n_a entries, 1/(e_size * kappa_h) (kappa = 1 outside CPML).
 * Replaces: the grid sizes folded into the coefficients
 * (calculation_param.cpp:235-263) and the kappa division of
 * PML::correctCoefficientX/Y/Z (src/boundary/pml.cpp:286-524). */
xfd_status xfd_set_curl_factors(xfd_engine* e, const double* const fe[3], const double* const fh[3]);

/* One CPML slab (one PML boundary).  E corrections act on layers
 * [e_start, e_start+thickness) of the slab axis, H corrections on
 * [h_start, h_start+thickness); a_*, b_* have `thickness` entries indexed by
 * layer.  Slabs are applied in the order they are added.
 * Replaces: PML::generateDomainCorrector (src/boundary/pml.cpp:246-284) and
 * PMLCorrector<xyz>::correctE/correctH (src/include/boundary/pml_corrector.h:178-382). */
typedef struct {
  int32_t axis;
  int32_t negative;
  int32_t thickness;
  int32_t e_start, h_start;
  const double *a_e, *b_e, *a_h, *b_h;
} xfd_cpml_slab;
xfd_status xfd_add_cpml(xfd_engine* e, const xfd_cpml_slab* slab);

/* TFSF3D plane-wave source.  e_inc (n_steps x aux) and h_inc
 * (n_steps x (aux-1)) are the FP64 1-D incident grid for every step; p_int[a]
 * (box size + 1 entries) and p_half[a] (box size + 2) the projections.
 * Replaces: TFSF3D::generateCorrector (src/waveform_source/tfsf_3d.cpp:21-45),
 * TFSF3DCorrector::correctE/correctH (src/waveform_source/tfsf_corrector.cpp:177-232). */
typedef struct {
  int32_t box_s[3], box_e[3];
  int32_t aux;
  const double* e_inc;
  const double* h_inc;
  const double* p_int[3];
  const double* p_half[3];
  double ca[3], cb[3];
  double te[3], th[3];
} xfd_tfsf_desc;
xfd_status xfd_set_tfsf(xfd_engine* e, const xfd_tfsf_desc* tfsf);
/* The same source on one x-slab of a lattice decomposed along x (the slab
 * decomposition driven by xfdtd_core_b200/slab.py, one engine per slab with a
 * ghost cell on each interior side): `tfsf` describes it on the global lattice
 * (box x coordinates global, projections and incident grid unchanged), and
 * plane 0 of this engine is global plane x_offset.  Every face pass is cut to
 * the nodes of this engine's lattice that it corrects, ghost cells included.
 * Replaces: the reference's cut of TFSF3D by the domain a process runs on
 * (TFSF3D::generateCorrector, src/waveform_source/tfsf_3d.cpp:21-33). */
xfd_status xfd_set_tfsf_slab(xfd_engine* e, const xfd_tfsf_desc* tfsf, int32_t x_offset);

/* Lumped current source on a box of E_comp nodes [box_s, box_e): per step
 * E += coff[node] * waveform[t].  coff is box-shaped (k fastest); waveform has
 * n_steps entries.  Replaces: CurrentSource::generateCorrector
 * (src/object/lumped_element/current_source.cpp:198-222) and
 * CurrentSourceCorrector::correctE (src/object/lumped_element/lumped_element_corrrector.cpp:24-37). */
xfd_status xfd_add_current_source(xfd_engine* e, int32_t comp, const int32_t box_s[3],
                                  const int32_t box_e[3], const double* coff,
                                  const double* waveform);

/* Lumped inductor on a box of E_comp nodes [box_s, box_e): after the E update
 * and the current sources, E += cecjc[node] * J[node], then
 * J[node] += cjcec[node] * E[node]; J (FP64) starts at zero and is part of the
 * saved state.  cecjc and cjcec are box-shaped (k fastest).  Added before the
 * first step.  The voltage source (the current-source form above), resistor
 * and capacitor are coefficient changes and source terms only.
 * Replaces: Inductor::generateCorrector (src/object/lumped_element/inductor.cpp:111-135)
 * and InductorCorrector::correctE (src/object/lumped_element/lumped_element_corrrector.cpp:42-99). */
xfd_status xfd_add_inductor(xfd_engine* e, int32_t comp, const int32_t box_s[3],
                            const int32_t box_e[3], const double* cecjc, const double* cjcec);

/* Dispersive (ADE) E nodes on a compacted list.  kind 0 = modified Lorentz
 * (J, J_prev, E_prev), 1 = Drude, 2 = Debye.  mat_coeff holds, per material,
 * 2 + 7*n_poles doubles: c_e_j_sum, c_e_e_prev, then per pole
 * (c_j_j, c_j_j_prev, c_j_e_next, c_j_e, c_j_e_prev, c_j_sum_j, c_j_sum_j_prev).
 * Entry n updates component comp[n] at lattice node (i,j,k) = node[3n..3n+2]
 * with material material[n].  The E coefficients of these nodes must already
 * be the overwritten ADE ones in the class table.
 * Replaces: Simulation::buildDispersiveSpace (src/simulation/simulation.cpp:745-829)
 * and MLorentzUpdator / DrudeADEUpdator3D / DebyeADEUpdator3D::updateE
 * (src/updator/m_lor_ade_updator.cpp:21-140,
 *  src/include/updator/ade_updator/template_ade_update_scheme.h:14-88). */
typedef struct {
  int32_t kind;
  int32_t n_poles;
  int32_t n_materials;
  const double* mat_coeff;
  int64_t n_entries;
  const uint8_t* comp;
  const int32_t* node;
  const uint8_t* material;
} xfd_ade_desc;
xfd_status xfd_set_ade(xfd_engine* e, const xfd_ade_desc* ade);

/* Frequency-domain NF2FF on the six Huygens faces.  Face d (XN XP YN YP ZN ZP)
 * covers nodes [task_s[d], task_e[d]) (empty when any extent is <= 0).
 * te / th are the FP64 phasors dt*exp(-j 2 pi f (t+1) dt) and
 * dt*exp(-j 2 pi f (t+1/2) dt), laid out (n_freq, n_steps, re/im).  Each step
 * adds `scale` times the step's term (scale = n_freq reproduces the
 * reference's per-step nF-fold accumulation).  Surface samples are batched
 * `batch` steps before the FP64 DFT accumulation.
 * Replaces: NFFFTFrequencyDomain::update (src/nffft/nffft_frequency_domain.cpp:45-53)
 * -> FDPlaneData::update/calculateJ/calculateM (src/nffft/nffft_fd_data_update.cpp:6-122). */
typedef struct {
  int32_t n_freq;
  int32_t batch;
  int32_t task_s[6][3];
  int32_t task_e[6][3];
  const double* te;
  const double* th;
  double scale;
} xfd_nf2ff_desc;
xfd_status xfd_set_nf2ff(xfd_engine* e, const xfd_nf2ff_desc* nf);

/* Accumulated J/M surface currents, complex interleaved, laid out
 * [freq][face][quantity ja jb ma mb][face nodes, k fastest].  `count` gets the
 * number of complex values.  Flushes a partial sample batch first.
 * Replaces: FDPlaneData's _ja/_jb/_ma/_mb arrays (src/nffft/nffft_fd_data.cpp:21-63). */
xfd_status xfd_get_nf2ff(xfd_engine* e, double* out, int64_t capacity, int64_t* count);

/* Far-field potentials of the accumulated surface currents, computed on the
 * GPU for n_angles (theta[a], phi[a]) pairs and every NF2FF frequency:
 * out = complex interleaved [freq][a_theta, f_phi, a_phi, f_theta][angle]
 * (n_freq * 4 * n_angles complex values).  freqs: the NF2FF frequencies (Hz),
 * n_freq of them; node_e / node_h / size_e: per axis the grid's node
 * coordinates (n+1), cell-centre coordinates (n) and cell sizes (n).
 * Replaces: FDPlaneData::getPotential / calculatePotential
 * (src/nffft/nffft_fd_data_process.cpp:15-144) as called by
 * NFFFTFrequencyDomain::processFarField (src/nffft/nffft_frequency_domain.cpp:103-129). */
typedef struct {
  int32_t n_angles;
  const double* theta;   /* host, n_angles */
  const double* phi;     /* host, n_angles */
  int32_t n_freq;
  const double* freqs;   /* host, n_freq */
  double origin[3];
  const double* node_e[3];
  const double* node_h[3];
  const double* size_e[3];
} xfd_far_field_desc;
xfd_status xfd_nf2ff_far_field(xfd_engine* e, const xfd_far_field_desc* d, double* out,
                               int64_t capacity);

/* Time-domain NF2FF for one observation direction.  Per step and Huygens
 * point (faces as in xfd_nf2ff_desc; points face by face XN..ZP, k fastest),
 * the change since the previous step of the surface-centre tangential E and
 * H, times the point's face-cell area ds, is added to the retarded-time bins
 * nn, nn + 1 (linear weights) of six potentials, nn + f = delay + 1/2 + t for
 * E and delay + t for H; delay = (the surface's largest projected distance -
 * the point's) / (c dt), computed by the caller.  xfd_get_nf2ff_td returns
 * the raw sums, 6 x n_bins doubles: W_x W_y W_z (from H) then U_x U_y U_z
 * (from E).
 * Replaces: NFFFTTimeDomain::update -> TDPlaneData::update
 * (src/nffft/nfffft_time_domain.cpp:80-96, src/include/nffft/nffft_td_data.h:169-240). */
typedef struct {
  int32_t task_s[6][3], task_e[6][3];
  const double* delay;  /* P values */
  const double* ds;     /* P values */
  int64_t n_bins;
} xfd_nf2ff_td_desc;

xfd_status xfd_set_nf2ff_td(xfd_engine* e, const xfd_nf2ff_td_desc* d);
xfd_status xfd_get_nf2ff_td(xfd_engine* e, double* out, int64_t capacity, int64_t* count);

/* Weighted probe: every step t, value = sum_q weight[q] F_comp[q](node q)
 * (comp 0..5 = Ex..Hz; node = (i, j, k), 3 per entry), reduced in FP64 into
 * row t of the probe's series.  xfd_get_probe copies the n_steps values.
 * Replaces: VoltageMonitor::update and CurrentMonitor::update
 * (src/monitor/voltage_monitor.cpp:198-235, src/monitor/current_monitor.cpp:253-379),
 * whose index ranges and weights the host computes. */
xfd_status xfd_add_probe(xfd_engine* e, int64_t n, const int32_t* comp, const int32_t* node,
                         const double* weight, int32_t* id);
xfd_status xfd_get_probe(xfd_engine* e, int32_t id, double* out, int64_t capacity,
                         int64_t* count);

/* Movie monitor: every `interval` steps (from step 0) the box [box_s, box_e)
 * of `field` is recorded into a device frame store.
 * Replaces: MovieMonitor::update -> FieldMonitor::output
 * (src/monitor/movie_monitor.cpp:26-34, src/monitor/field_monitor.cpp:82-96). */
xfd_status xfd_add_movie(xfd_engine* e, int32_t field, const int32_t box_s[3],
                         const int32_t box_e[3], int32_t interval, int32_t* id);

/* Copies the frames recorded so far (in the engine precision) into `out`.
 * Replaces: Monitor::output (src/monitor/monitor.cpp:42-54). */
xfd_status xfd_get_movie_frames(xfd_engine* e, int32_t id, void* out, int64_t capacity_bytes,
                                int64_t* n_frames);

/* Field exchange in the reference shapes, elements in the engine precision
 * (double for XFD_FP64, float for XFD_FP32).  fields[0..5] = Ex..Hz.
 * Replaces: direct access to EMF (include/xfdtd/electromagnetic_field/electromagnetic_field.h:18-126). */
xfd_status xfd_upload_fields(xfd_engine* e, const void* const fields[6]);
xfd_status xfd_download_fields(xfd_engine* e, void* const fields[6]);

/* One field component, `field` 0..5, in its reference shape. */
xfd_status xfd_download_field(xfd_engine* e, int32_t field, void* out);

/* Advances n_steps time steps (captured as CUDA graphs where possible).
 * Asynchronous with respect to the host; xfd_sync waits.
 * Replaces: Simulation::run() -> Domain::run (src/simulation/simulation.cpp:291-317,
 * src/domain/domain.cpp:45-138). */
xfd_status xfd_run(xfd_engine* e, int64_t n_steps);
xfd_status xfd_sync(xfd_engine* e);

/* Steps completed (queued) so far. */
int64_t xfd_current_step(const xfd_engine* e);

/* Engine options: "graph" (0/1, default 1), "graph_chunk" (steps per graph,
 * default 32), "kernel" (the Yee sweep: 0 = split H/E sweeps, 1 = fused
 * H-then-E sweep, 2 = fused sweep with its per-plane inputs staged by TMA,
 * 3 = split sweeps marching along x, 4 = the same with TMA-staged planes,
 * 5 = fused marching sweep with overlapped tiles and TMA-staged planes,
 * 6 = 5 with a two-nodes-per-thread form in the CPML-free interior,
 * 7 = the fused H-then-E sweep of the CPML-free interior box with ping-pong
 * buffers beside the split marching sweeps of the CPML tiles; default 7, or 0
 * on lattices whose marching tiles number fewer than two per SM),
 * "ichunk" (planes per CTA of the fused sweeps, default 32), "march_ichunk"
 * (planes per CTA of the split marching sweeps, default 16), and the forms
 * of sweep 4: "march_concurrent" (launches of a phase on four streams,
 * default 1), "march_split_axes" (CPML tiles in lists by slab axis, default
 * 1), "march_cp_stages" (single-axis lists with fewer stages, default 1),
 * "march_wide" (two-rows-per-thread interior form, default 0),
 * "march_shift" (tile grid moved to the CPML layers along k, default 0;
 * sweep 7 always moves it along j and i), and of sweep 0: "pdl"
 * (programmatic dependent launch of the step's kernels, default 1).  Every
 * sweep computes the same update; they differ in speed only.
 * Failure detection: "stage_wait_cycles" (cycles a TMA-staged sweep (3..7)
 * waits for one staged plane before the CTA gives up, drains its loads in
 * flight and returns; the next xfd_sync reports XFD_ERR_TIMEOUT; 0 = the
 * default, about 2 s; batched engines take the value they had at
 * xfd_batch_create) and "watchdog_interval" (K > 0: every K steps a scan of
 * the six fields for NaN / Inf; the next xfd_sync reports XFD_ERR_NUMERIC;
 * default 0 = off; not run by xfd_batch_run).  An engine whose sweep gave up
 * stays stopped (every later sweep CTA returns at once); the CUDA context
 * stays usable, so a new engine can take over. */
xfd_status xfd_set_option(xfd_engine* e, const char* name, int64_t value);
/* Current value of an option of xfd_set_option. */
xfd_status xfd_get_option(const xfd_engine* e, const char* name, int64_t* value);

/* The CUDA stream the engine launches on (a cudaStream_t), for callers that
 * time the engine with events on that stream. */
void* xfd_stream(xfd_engine* e);

/* Number of kernel launches per time step of the current configuration. */
int32_t xfd_launches_per_step(const xfd_engine* e);

/* Algorithmic DRAM bytes per time step of the stencil sweep (fields read and
 * written once, class index, CPML auxiliaries) -- the roofline numerator. */
int64_t xfd_stencil_bytes_per_step(const xfd_engine* e);

/* Algorithmic DRAM bytes per time step of the whole step: the stencil bytes
 * above plus the ADE currents (J, and for the modified-Lorentz form J_prev and
 * E_prev, read and written once per dispersive entry), the TFSF face passes
 * (each corrected node read and written once) and the NF2FF (four FP64
 * samples written per surface point, and the complex FP64 accumulators read
 * and written once per DFT batch).  No credit for reuse across steps. */
int64_t xfd_algorithmic_bytes_per_step(const xfd_engine* e);

/* ---- Allocation-free NF2FF step -------------------------------------------
 * No counterpart in the reference: an addition of this library for callers
 * that cannot allocate device memory -- an FDTD loop embedded in a larger GPU
 * application whose device memory is all owned by its own pool or a fixed
 * arena, where a cudaMalloc would fail or would synchronise the device in the
 * middle of the caller's time loop.  It folds ONE time step of the Huygens-
 * surface fields into the NF2FF frequency-domain surface currents, exactly
 * what the engine's NF2FF does per step (xfd_set_nf2ff), but on the caller's
 * arrays and without allocating: it calls no cudaMalloc or cudaFree and no
 * allocating library routine.  The per-step samples go to a fixed scratch
 * array of 4 x XFD_NF2FF_STATIC_MAX_POINTS doubles (4 MiB) compiled into the
 * library, which every GPU that loads the library holds until exit.
 *   - The first call on a device looks up that array's device address
 *     (cudaGetSymbolAddress) with the device current; make that first call
 *     before any stream capture.  The address is kept per CUDA context, so
 *     the first call after a cudaDeviceReset looks it up again.
 *   - All calls on a device share the one scratch array: calls whose kernels
 *     overlap on the GPU (different streams or host threads) race and corrupt
 *     each other's samples -- serialise them.
 *   - Nothing in the scratch has to start at zero (each call writes every
 *     entry it reads).  `acc` is accumulated into: zero it before the first
 *     step, as the engine zeroes its own accumulator.
 *   - Surfaces of more than XFD_NF2FF_STATIC_MAX_POINTS points, or more than
 *     XFD_NF2FF_STATIC_MAX_FREQ frequencies, are rejected with
 *     XFD_ERR_UNSUPPORTED / XFD_ERR_INVALID_ARGUMENT and a message in
 *     xfd_last_error(NULL); nothing is launched then. */
#define XFD_NF2FF_STATIC_MAX_POINTS 131072
#define XFD_NF2FF_STATIC_MAX_FREQ 1024

typedef struct {
  int32_t nx, ny, nz;     /* grid cells */
  int32_t precision;      /* element type of the fields: XFD_FP64 or XFD_FP32 */
  const void* fields[6];  /* device arrays Ex Ey Ez Hx Hy Hz in the reference
                             component shapes, C order (Ex: nx x (ny+1) x (nz+1),
                             Hx: (nx+1) x ny x nz, ...) */
  int32_t n_freq;
  int32_t task_s[6][3];   /* Huygens faces, as in xfd_nf2ff_desc */
  int32_t task_e[6][3];
  const double* te;       /* device, n_freq x n_steps complex (re, im): E-time phasors */
  const double* th;       /* device, n_freq x n_steps complex: H-time phasors */
  int64_t n_steps;
  int64_t step;           /* time index t of this step, 0 <= step < n_steps */
  double scale;
  double* acc;            /* device, n_freq x 4 x P complex, accumulated in place
                             (P = points of the six faces, face by face) */
  double* acc_comp;       /* optional device array shaped like acc (zeroed before
                             the first step) for compensated accumulation: each
                             step's rounding error goes there, and the surface
                             current is acc + acc_comp.  NULL: plain sums. */
} xfd_nf2ff_step_desc;

/* Queues the step on `stream` (a cudaStream_t; NULL = legacy default). */
xfd_status xfd_nf2ff_step_static(const xfd_nf2ff_step_desc* d, void* stream);

/* ---- Saved states ----------------------------------------------------------
 * No counterpart in the reference (whose TimeParam has a start step but no
 * saved field state).  A slot holds a device copy of what the next step
 * reads: the six fields, the CPML auxiliaries, the ADE currents and the step
 * counter.  Movie frames are outputs and are not rewound.  An engine with a
 * frequency- or time-domain NF2FF surface refuses xfd_checkpoint_load
 * (XFD_ERR_UNSUPPORTED): its running DFT sums and per-step sample ring cover
 * the steps already taken and cannot be rewound.
 * Slots are engine-owned device memory (0 <= slot < 4096); saving over a
 * slot reuses it.  Loading a slot saved under another configuration (CPML
 * slabs, ADE) is rejected (XFD_ERR_STATE). */
xfd_status xfd_checkpoint_save(xfd_engine* e, int32_t slot);
xfd_status xfd_checkpoint_load(xfd_engine* e, int32_t slot);
xfd_status xfd_checkpoint_drop(xfd_engine* e, int32_t slot);
/* Step at which `slot` was saved, -1 if empty. */
int64_t xfd_checkpoint_step(const xfd_engine* e, int32_t slot);

/* ---- Adjoint gradient ------------------------------------------------------
 * No counterpart in the reference (no gradient path): the discrete adjoint
 * of the time step -- the exact transpose of the E/H updates with their CPML
 * auxiliaries, run backward in time (TFSF faces and lumped sources are
 * state-independent terms and have none).  Engines with ADE media, an NF2FF
 * surface or movies are rejected (XFD_ERR_UNSUPPORTED).
 *
 * xfd_adjoint_run advances n_steps from the current state (N = n_steps),
 * saving the state every checkpoint_interval (K) steps and recording E
 * component obj_field over the node box [obj_s, obj_e) after every step.
 * It then calls `objective` once with that record (row n = after n+1 steps,
 * points in box order, k fastest), which returns J in *value and dJ/drecord
 * in d_record (same shape); return nonzero to abort (XFD_ERR_NUMERIC).  The
 * reverse pass recomputes each K-step segment from its saved state (memory
 * holds ceil(N/K) + 1 states and K + 1 design-box rows) and returns in
 * `sens` (2 x 3 x n_design doubles, n_design = nodes of [design_s,
 * design_e), k fastest):
 *   sens[0][c][p] = sum_{m=1..N} lam_c^m(p) E_c^{m-1}(p)
 *   sens[1][c][p] = sum_{m=1..N} lam_c^m(p) E_c^m(p)
 * with lam^m = dJ/dE^m, the total derivative of J with respect to the E field
 * after m steps (through every later step).  At a node where the step is
 * E^m = ca E^{m-1} + cb C^m (main range, outside CPML layers, TFSF faces and
 * sources), C^m = (E^m - ca E^{m-1}) / cb, so for a parameter p of the
 * node's (ca, cb):
 *   dJ/dp = (ca' - ca cb'/cb) sens[0] + (cb'/cb) sens[1]     (' = d/dp).
 * On return the engine holds the state after the N forward steps. */
typedef int32_t (*xfd_objective_fn)(void* user, int64_t n_steps, int64_t n_points,
                                    const double* record, double* d_record, double* value);

typedef struct {
  int64_t n_steps;
  int32_t checkpoint_interval;
  int32_t forward_only;               /* 1: record and evaluate J only (no states saved,
                                         no reverse pass, sens unused) */
  int32_t obj_field;                  /* 0..2: Ex, Ey, Ez */
  int32_t obj_s[3], obj_e[3];         /* objective node box [s, e) */
  int32_t design_s[3], design_e[3];   /* design node box [s, e) */
  xfd_objective_fn objective;
  void* user;
} xfd_adjoint_desc;

xfd_status xfd_adjoint_run(xfd_engine* e, const xfd_adjoint_desc* d, double* value,
                           double* sens);

/* ---- Batched simulations ---------------------------------------------------
 * No counterpart in the reference (which runs one Simulation per process):
 * many independent simulations of uneven grid sizes -- design variants,
 * incidence angles -- advanced together on one GPU.  Each is an engine set
 * up as usual (xfd_create, classes, curl factors, CPML, TFSF, fields); the
 * batch advances them with a time step of all of them one launch of a
 * persistent kernel over a device work queue (every tile, lattice-face block
 * and TFSF block of the step, with bounded per-engine dependency waits; the
 * option "queue" = 0 gives a launch per phase and sweep form instead),
 * captured as CUDA graphs.
 * Per engine the arithmetic and order are those of xfd_run with the default
 * sweep.  Engines with ADE media, lumped sources, movies or an NF2FF surface
 * are rejected (XFD_ERR_UNSUPPORTED); all engines share one device and one
 * precision.  The batch borrows the engines: destroy it before them, and do
 * not call xfd_run on them while the batch runs.  After xfd_batch_run each
 * engine's step count has advanced and its own stream is ordered after the
 * batch, so xfd_download_fields / xfd_sync on an engine see the results. */
typedef struct xfd_batch xfd_batch;

xfd_status xfd_batch_create(xfd_engine* const* engines, int32_t n, xfd_batch** out);
void xfd_batch_destroy(xfd_batch* b);
/* Message of the last failure on `b` (NULL: of a failed xfd_batch_create). */
const char* xfd_batch_last_error(const xfd_batch* b);

/* Advances every engine of the batch n_steps (asynchronous; xfd_batch_sync
 * waits and reports device-side errors of any engine). */
xfd_status xfd_batch_run(xfd_batch* b, int64_t n_steps);
xfd_status xfd_batch_sync(xfd_batch* b);

/* Options: "graph" (0/1, default 1), "graph_chunk" (steps per graph, default
 * 32), "march_ichunk" (x planes per CTA, the tile depth, default 16),
 * "queue" (0/1, default 1: the persistent work-queue launch), "concurrent"
 * (0/1, default 1: the launch-per-phase form runs its single-axis CPML tile
 * lists on three side streams beside the other forms), "tile_rows"
 * (rows per tile, 8 or 16; 16 needs the queue form), "queue_wait_cycles"
 * (cycles a queue item waits for the items it depends on before the batch
 * reports XFD_ERR_TIMEOUT; 0: the stage-wait default, about 2 s),
 * "queue_stall_test" (1: one item waits for a count that is never reached,
 * to test that timeout) and "autotune" (K > 0: the next xfd_batch_run of at
 * least 12 (1 + K) steps times K steps of each of 12 candidates inside the
 * run and keeps the fastest, setting "queue", "tile_rows" and "march_ichunk"
 * -- the queue form at tile rows 8 and 16 and the launch per phase at 8, each
 * at tile depths 8, 16, 32, 64; neither form nor tiling changes the
 * results). */
xfd_status xfd_batch_set_option(xfd_batch* b, const char* name, int64_t value);
xfd_status xfd_batch_get_option(const xfd_batch* b, const char* name, int64_t* value);

/* The last autotuning: candidate tile depths and their ms per batch step. */
xfd_status xfd_batch_tuning(const xfd_batch* b, int32_t* depth, double* ms_per_step,
                            int32_t capacity, int32_t* count);
/* The same with each candidate's form (1: queue) and tile rows. */
xfd_status xfd_batch_tuning_shapes(const xfd_batch* b, int32_t* queue, int32_t* rows,
                                   int32_t* depth, double* ms_per_step, int32_t capacity,
                                   int32_t* count);

int32_t xfd_batch_size(const xfd_batch* b);
/* Kernel launches per batch step (after the first xfd_batch_run). */
int32_t xfd_batch_launches_per_step(const xfd_batch* b);
/* The CUDA stream the batch launches on (a cudaStream_t). */
void* xfd_batch_stream(xfd_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* XFD_ENGINE_H_ */
