/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  PARITY UNPINNED.
 *
 * CPU restatement, in plain C (FP64, no FMA contraction), of the per-time-step
 * arithmetic of EMinsight/XFDTD_CORE's 3-D FDTD hot path.  The CUDA
 * engine's parity tests compare against it, and it is the timed CPU baseline;
 * nothing in the product links it.  The reference ships no golden vectors and cannot be
 * compiled here (it needs xtensor/xtl, which are absent), so this restatement
 * is not pinned to outputs of the reference itself: every routine instead
 * cites the reference lines it follows.
 *
 * Arrays use the reference's shapes and row-major (i, j, k) layout:
 *   Ex(nx, ny+1, nz+1) Ey(nx+1, ny, nz+1) Ez(nx+1, ny+1, nz)
 *   Hx(nx+1, ny, nz)   Hy(nx, ny+1, nz)   Hz(nx, ny, nz+1)
 * and the 18 coefficient arrays have the shape of their field
 * (src/simulation/simulation.cpp:514-528,
 *  include/xfdtd/calculation_param/fdtd_update_coefficient.h:102-121).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t idx_t;

/* One field-shaped 3-D array. */
typedef struct {
  double *p;
  idx_t n[3];
} orc_arr;

#define AT(a, i, j, k) ((a).p[((idx_t)(i) * (a).n[1] + (idx_t)(j)) * (a).n[2] + (idx_t)(k)])

/* Fields and the 18 Yee coefficients.  Component order x, y, z. */
typedef struct {
  idx_t nx, ny, nz;
  orc_arr e[3], h[3];
  orc_arr ce[3];      /* cexe ceye ceze */
  orc_arr ceh_a[3];   /* coefficient of E_c w.r.t. H_a (a = tangential A axis of c):
                         cexhy ceyhz cezhx */
  orc_arr ceh_b[3];   /* w.r.t. H_b: cexhz ceyhx cezhy */
  orc_arr ch[3];      /* chxh chyh chzh */
  orc_arr che_a[3];   /* chxey chyez chzex */
  orc_arr che_b[3];   /* chxez chyex chzey */
} orc_yee;

/* Tangential axes: X -> (Y, Z), Y -> (Z, X), Z -> (X, Y)
 * (include/xfdtd/coordinate_system/coordinate_system.h:192-203). */
static inline int tan_a(int c) { return (c + 1) % 3; }
static inline int tan_b(int c) { return (c + 2) % 3; }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * Yee H update: BasicUpdator::updateH (src/updator/basic_updator.cpp:23-36)
 * -> update<H, xyz> (src/include/updator/update_scheme.h:64-108) with
 * hNext (update_scheme.h:57-62):
 *   H_c = ch*H_c + che_a*(E_a[c_b + 1] - E_a) + che_b*(E_b[c_a + 1] - E_b)
 * over i in [0,nx), j in [0,ny), k in [0,nz) for all three components
 * (include/xfdtd/util/fdtd_basic.h:175-195).
 * ---------------------------------------------------------------------- */
void orc_update_h(const orc_yee *y) {
  const idx_t nx = y->nx, ny = y->ny, nz = y->nz;
  for (int c = 0; c < 3; ++c) {
    const int a = tan_a(c), b = tan_b(c);
    const orc_arr F = y->h[c], Ea = y->e[a], Eb = y->e[b];
    const orc_arr C0 = y->ch[c], Ca = y->che_a[c], Cb = y->che_b[c];
#pragma omp parallel for schedule(static)
    for (idx_t i = 0; i < nx; ++i) {
      for (idx_t j = 0; j < ny; ++j) {
        for (idx_t k = 0; k < nz; ++k) {
          idx_t p[3] = {i, j, k};
          /* field_a at (a, b+1, c): step +1 along the tangential B axis. */
          idx_t qa[3] = {i, j, k};
          qa[b] += 1;
          /* field_b at (a+1, b, c): step +1 along the tangential A axis. */
          idx_t qb[3] = {i, j, k};
          qb[a] += 1;
          const double ea_p = AT(Ea, p[0], p[1], p[2]);
          const double ea_q = AT(Ea, qa[0], qa[1], qa[2]);
          const double eb_p = AT(Eb, p[0], p[1], p[2]);
          const double eb_q = AT(Eb, qb[0], qb[1], qb[2]);
          double *f = &AT(F, i, j, k);
          *f = AT(C0, i, j, k) * *f + AT(Ca, i, j, k) * (ea_q - ea_p) +
               AT(Cb, i, j, k) * (eb_q - eb_p);
        }
      }
    }
  }
}

/* E update ranges (src/updator/basic_updator_3d.cpp:38-69): the start index
 * of both tangential axes is bumped to 1, so tangential E on the outer PEC
 * walls is never updated. */
static void e_range(const orc_yee *y, int c, idx_t s[3], idx_t e[3]) {
  s[0] = 0; s[1] = 0; s[2] = 0;
  e[0] = y->nx; e[1] = y->ny; e[2] = y->nz;
  s[tan_a(c)] = 1;
  s[tan_b(c)] = 1;
}

/* ------------------------------------------------------------------------
 * Yee E update: BasicUpdator3D::updateE (basic_updator_3d.cpp:38-77) ->
 * update<E, xyz> with eNext (update_scheme.h:26-31):
 *   E_c = ce*E_c + ceh_a*(H_a - H_a[c_b - 1]) + ceh_b*(H_b - H_b[c_a - 1])
 * ---------------------------------------------------------------------- */
void orc_update_e(const orc_yee *y) {
  for (int c = 0; c < 3; ++c) {
    const int a = tan_a(c), b = tan_b(c);
    const orc_arr F = y->e[c], Ha = y->h[a], Hb = y->h[b];
    const orc_arr C0 = y->ce[c], Ca = y->ceh_a[c], Cb = y->ceh_b[c];
    idx_t s[3], e[3];
    e_range(y, c, s, e);
#pragma omp parallel for schedule(static)
    for (idx_t i = s[0]; i < e[0]; ++i) {
      for (idx_t j = s[1]; j < e[1]; ++j) {
        for (idx_t k = s[2]; k < e[2]; ++k) {
          idx_t qa[3] = {i, j, k};
          qa[b] -= 1;
          idx_t qb[3] = {i, j, k};
          qb[a] -= 1;
          const double ha_p = AT(Ha, i, j, k);
          const double ha_q = AT(Ha, qa[0], qa[1], qa[2]);
          const double hb_p = AT(Hb, i, j, k);
          const double hb_q = AT(Hb, qb[0], qb[1], qb[2]);
          double *f = &AT(F, i, j, k);
          *f = AT(C0, i, j, k) * *f + AT(Ca, i, j, k) * (ha_p - ha_q) +
               AT(Cb, i, j, k) * (hb_p - hb_q);
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------
 * ADE E update.  Storage is full-grid (nx, ny, nz[, P]) like the reference
 * (src/material/ade_method/m_lor_ade_method.cpp:43-64); cells that are not
 * dispersive carry zero coefficients, which leaves the plain Yee result.
 * kind 0: MLorentzUpdator::updateE/updateJ/calculateJSum/recordEPrevious
 *         (src/updator/m_lor_ade_updator.cpp:21-140)
 * kind 1: Drude (src/updator/ade_updator/drude_ade_updator.cpp:21-39 with
 *         TemplateADEUpdateScheme::updateE,
 *         src/include/updator/ade_updator/template_ade_update_scheme.h:14-88;
 *         ePrevious/coeffEPrev are 0, drude_ade_updator.h:29-39)
 * kind 2: Debye (src/updator/ade_updator/debye_ade_updator.cpp:33-51)
 * ---------------------------------------------------------------------- */
typedef struct {
  int kind;
  idx_t np;
  double *cjj, *cjjp, *cjen, *cje, *cjep, *cjsumj, *cjsumjp; /* (nx,ny,nz,np) */
  double *cejsum, *ceep;                                      /* (nx,ny,nz) */
  double *eprev[3];                                           /* (nx,ny,nz) */
  double *j[3], *jprev[3];                                    /* (nx,ny,nz,np) */
} orc_ade;

void orc_update_e_ade(const orc_yee *y, const orc_ade *ad) {
  const idx_t ny = y->ny, nz = y->nz, np = ad->np;
  for (int c = 0; c < 3; ++c) {
    const int a = tan_a(c), b = tan_b(c);
    const orc_arr F = y->e[c], Ha = y->h[a], Hb = y->h[b];
    const orc_arr C0 = y->ce[c], Ca = y->ceh_a[c], Cb = y->ceh_b[c];
    idx_t s[3], e[3];
    e_range(y, c, s, e);
    double *J = ad->j[c], *Jp = ad->jprev[c], *Ep = ad->eprev[c];
#pragma omp parallel for schedule(static)
    for (idx_t i = s[0]; i < e[0]; ++i) {
      for (idx_t j = s[1]; j < e[1]; ++j) {
        for (idx_t k = s[2]; k < e[2]; ++k) {
          const idx_t cell = (i * ny + j) * nz + k;
          idx_t qa[3] = {i, j, k};
          qa[b] -= 1;
          idx_t qb[3] = {i, j, k};
          qb[a] -= 1;
          /* calculateJSum */
          double j_sum = 0;
          for (idx_t p = 0; p < np; ++p) {
            if (ad->kind == 0) {
              j_sum += ad->cjsumj[cell * np + p] * J[cell * np + p] +
                       ad->cjsumjp[cell * np + p] * Jp[cell * np + p];
            } else {
              j_sum += ad->cjsumj[cell * np + p] * J[cell * np + p];
            }
          }
          const double e_prev = (ad->kind == 0) ? Ep[cell] : 0.0;
          const double c_ep = (ad->kind == 0) ? ad->ceep[cell] : 0.0;
          double *f = &AT(F, i, j, k);
          const double e_cur = *f;
          const double en = AT(C0, i, j, k) * *f +
                            AT(Ca, i, j, k) * (AT(Ha, i, j, k) - AT(Ha, qa[0], qa[1], qa[2])) +
                            AT(Cb, i, j, k) * (AT(Hb, i, j, k) - AT(Hb, qb[0], qb[1], qb[2]));
          *f = c_ep * e_prev + en + ad->cejsum[cell] * j_sum;
          const double e_next = *f;
          /* updateJ */
          for (idx_t p = 0; p < np; ++p) {
            const idx_t q = cell * np + p;
            if (ad->kind == 0) {
              const double jn = ad->cjen[q] * e_next + ad->cje[q] * e_cur +
                                ad->cjep[q] * e_prev + ad->cjj[q] * J[q] +
                                ad->cjjp[q] * Jp[q];
              Jp[q] = J[q];
              J[q] = jn;
            } else if (ad->kind == 1) {
              J[q] = ad->cjj[q] * J[q] + ad->cje[q] * (e_next + e_cur);
            } else {
              J[q] = ad->cjj[q] * J[q] + ad->cje[q] * (e_next - e_cur);
            }
          }
          /* recordEPrevious */
          if (ad->kind == 0) Ep[cell] = e_cur;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------
 * CPML slab.  PMLCorrector<xyz>::correctE/correctH
 * (src/include/boundary/pml_corrector.h:178-382) -> correctPML (:14-52).
 * One slab per PML boundary; `m` is its main axis; A, B its tangential axes.
 * psi / c_psi arrays are the reference's node-local slab arrays
 * (src/boundary/pml.cpp:286-524): E_A <- ea_psi_hb, E_B <- eb_psi_ha,
 * H_A <- ha_psi_eb, H_B <- hb_psi_ea.
 * ---------------------------------------------------------------------- */
typedef struct {
  int m;
  idx_t n;                        /* thickness */
  idx_t e_start, h_start;         /* global == node start indices */
  idx_t task_s[3], task_e[3];     /* the PML node task (x, y, z) */
  double *a_e, *b_e, *a_h, *b_h;  /* length n */
  orc_arr c_psi[4];               /* ea_hb, eb_ha, ha_eb, hb_ea */
  orc_arr psi[4];
} orc_pml;

static void pml_block(orc_arr F, orc_arr D, orc_arr CP, orc_arr P, const double *ca,
                      const double *cb, int m, int is_e, idx_t s[3], idx_t e[3],
                      idx_t start) {
  const int off = is_e ? -1 : 1;
#pragma omp parallel for schedule(static)
  for (idx_t i = s[0]; i < e[0]; ++i) {
    for (idx_t j = s[1]; j < e[1]; ++j) {
      for (idx_t k = s[2]; k < e[2]; ++k) {
        idx_t x[3] = {i, j, k};
        const idx_t cc = x[m];
        const double av = ca[cc - start];
        const double bv = cb[cc - start];
        idx_t l[3] = {i, j, k};
        l[m] = cc - start;
        idx_t q[3] = {i, j, k};
        q[m] = cc + off;
        const double dp = AT(D, i, j, k);
        const double dq = AT(D, q[0], q[1], q[2]);
        double *psi = &AT(P, l[0], l[1], l[2]);
        if (is_e) {
          *psi = bv * *psi + av * (dp - dq);
        } else {
          *psi = bv * *psi + av * (dq - dp);
        }
        AT(F, i, j, k) += AT(CP, l[0], l[1], l[2]) * *psi;
      }
    }
  }
}

void orc_pml_correct(const orc_yee *y, const orc_pml *pm, int is_e) {
  const int m = pm->m, A = tan_a(m), B = tan_b(m);
  idx_t s[3], e[3];
  for (int d = 0; d < 3; ++d) {
    s[d] = pm->task_s[d];
    e[d] = pm->task_e[d];
  }
  if (is_e) {
    idx_t off = 0;
    if (s[m] == 0) {  /* pml_corrector.h:197-208 */
      s[m] = 1;
      off = 1;
    }
    const idx_t start = pm->e_start;
    /* E_A: [a_s, a_e), [b_s, b_e + 1), [c_s, c_e + off) (:219-247) */
    idx_t ea[3] = {e[0], e[1], e[2]};
    ea[B] += 1;
    ea[m] += off;
    pml_block(y->e[A], y->h[B], pm->c_psi[0], pm->psi[0], pm->a_e, pm->b_e, m, 1, s, ea,
              start);
    /* E_B: [a_s, a_e + 1), [b_s, b_e), [c_s, c_e + off) (:257-286) */
    idx_t eb[3] = {e[0], e[1], e[2]};
    eb[A] += 1;
    eb[m] += off;
    pml_block(y->e[B], y->h[A], pm->c_psi[1], pm->psi[1], pm->a_e, pm->b_e, m, 1, s, eb,
              start);
  } else {
    const idx_t start = pm->h_start;
    /* H_A: [a_s, a_e + 1), [b_s, b_e), [c_s, c_e) (:316-343) */
    idx_t ha[3] = {e[0], e[1], e[2]};
    ha[A] += 1;
    pml_block(y->h[A], y->e[B], pm->c_psi[2], pm->psi[2], pm->a_h, pm->b_h, m, 0, s, ha,
              start);
    /* H_B: [a_s, a_e), [b_s, b_e + 1), [c_s, c_e) (:353-380) */
    idx_t hb[3] = {e[0], e[1], e[2]};
    hb[B] += 1;
    pml_block(y->h[B], y->e[A], pm->c_psi[3], pm->psi[3], pm->a_h, pm->b_h, m, 0, s, hb,
              start);
  }
}

/* ------------------------------------------------------------------------
 * TFSF3D face corrections: TFSF3DCorrector::correctE/correctH
 * (src/waveform_source/tfsf_corrector.cpp:177-232) -> correctTFSF
 * (src/include/waveform_source/tfsf_corrector.h:89-229) with the incident
 * interpolation exInc..hzInc (tfsf_corrector.cpp:16-122).
 * ---------------------------------------------------------------------- */
typedef struct {
  idx_t is, ie, js, je, ks, ke;   /* TFSF box [s, e) in global indices */
  idx_t nt, aux;
  const double *e_inc, *h_inc;    /* (nt, aux), (nt, aux - 1) */
  const double *p_int[3], *p_half[3];
  double ca[3], cb[3];            /* dt/(eps0 d), dt/(mu0 d) per axis */
  double te[3], th[3];            /* transform_e / transform_h */
  /* The lattice this oracle runs is the x-slab of the global one whose plane
   * 0 is global plane xo, nxl cells along x (xo = 0, nxl = nx: the whole
   * lattice).  Passes correct only the nodes of the slab, as the reference
   * cuts TFSF3D by the domain a process runs on (TFSF3D::generateCorrector,
   * src/waveform_source/tfsf_3d.cpp:21-33). */
  idx_t xo, nxl;
} orc_tfsf;

/* exInc..hzInc.  The axis whose index is shifted by +1 uses the half-cell
 * projection; H components subtract 0.5 and read h_inc. */
static double tfsf_inc(const orc_tfsf *t, int is_e, int comp, idx_t step, idx_t i,
                       idx_t j, idx_t k) {
  idx_t r[3] = {i - t->is, j - t->js, k - t->ks};
  double proj;
  if (is_e) {
    /* E_comp: half projection along comp, integer along the others. */
    r[comp] += 1;
    proj = 0;
    double parts[3];
    for (int d = 0; d < 3; ++d) parts[d] = (d == comp) ? t->p_half[d][r[d]] : t->p_int[d][r[d]];
    proj = parts[0] + parts[1] + parts[2];
    const idx_t index = (idx_t)proj;
    const double w = proj - (double)index;
    const double *row = t->e_inc + step * t->aux;
    return t->te[comp] * ((1 - w) * row[index] + w * row[index + 1]);
  }
  /* H_comp: integer projection along comp, half along the others, -0.5. */
  double parts[3];
  for (int d = 0; d < 3; ++d) {
    if (d != comp) r[d] += 1;
    parts[d] = (d == comp) ? t->p_int[d][r[d]] : t->p_half[d][r[d]];
  }
  proj = parts[0] + parts[1] + parts[2] - 0.5;
  const idx_t index = (idx_t)proj;
  const double w = proj - (double)index;
  const double *row = t->h_inc + step * (t->aux - 1);
  return t->th[comp] * ((1 - w) * row[index] + w * row[index + 1]);
}

/* One correctTFSF<direction, attribute, field_xyz> pass.  Indices are
 * global; the node corrected is written at local x = global x - xo when the
 * slab holds it (E_x, H_y, H_z: x < nxl; the others x <= nxl). */
static void tfsf_pass(const orc_yee *y, const orc_tfsf *t, idx_t step, int dir_axis,
                      int negative, int is_e, int field) {
  const int m = dir_axis, A = tan_a(m), B = tan_b(m);
  const int dual_field = (field == A) ? B : A;
  idx_t s[3] = {t->is, t->js, t->ks};
  idx_t e[3] = {t->ie, t->je, t->ke};
  /* offset_a / offset_b (tfsf_corrector.h:122-140): the node task equals the
   * TFSF task for one domain, so the extension always applies. */
  const int offset_a = ((is_e && field == B) || (!is_e && field == A)) ? 1 : 0;
  if (offset_a) e[A] += 1; else e[B] += 1;
  /* The corrected plane is the box start (negative faces) or end. */
  const idx_t cs = negative ? s[m] : e[m];
  s[m] = cs;
  e[m] = cs + 1;
  const int equation_flag = is_e ? 1 : -1;
  const int different_flag = (field == A) ? -1 : 1;
  const int direction_flag = negative ? -1 : 1;
  const double flag = (double)(equation_flag * different_flag * direction_flag);
  const double coeff = (is_e ? t->ca[m] : t->cb[m]) * flag;
  orc_arr F = is_e ? y->e[field] : y->h[field];
  const int on_cells = is_e ? field == 0 : field != 0;
  const idx_t x_end = on_cells ? t->nxl : t->nxl + 1;  /* local x range [0, x_end) */
  for (idx_t i = s[0]; i < e[0]; ++i) {
    /* x of the node this i corrects (a negative H face along x: one below) */
    const idx_t xc = i - ((negative && !is_e && m == 0) ? 1 : 0) - t->xo;
    if (xc < 0 || xc >= x_end) continue;
    for (idx_t j = s[1]; j < e[1]; ++j) {
      for (idx_t k = s[2]; k < e[2]; ++k) {
        idx_t x[3] = {i, j, k};
        if (negative) {
          idx_t q[3] = {i, j, k};
          q[m] -= 1;
          if (is_e) {
            const double v = tfsf_inc(t, 0, dual_field, step, q[0], q[1], q[2]);
            AT(F, i - t->xo, j, k) += v * coeff;
          } else {
            const double v = tfsf_inc(t, 1, dual_field, step, i, j, k);
            AT(F, q[0] - t->xo, q[1], q[2]) += v * coeff;
          }
        } else {
          const double v = tfsf_inc(t, is_e ? 0 : 1, dual_field, step, x[0], x[1], x[2]);
          AT(F, i - t->xo, j, k) += v * coeff;
        }
      }
    }
  }
}

void orc_tfsf_correct(const orc_yee *y, const orc_tfsf *t, idx_t step, int is_e) {
  /* Pass order of TFSF3DCorrector::correctE / correctH. */
  static const int e_passes[12][3] = {
      {0, 1, 2}, {0, 0, 2}, {1, 1, 2}, {1, 0, 2}, {2, 1, 1}, {2, 0, 1},
      {0, 1, 1}, {0, 0, 1}, {2, 1, 0}, {2, 0, 0}, {1, 1, 0}, {1, 0, 0}};
  static const int h_passes[12][3] = {
      {0, 1, 1}, {0, 0, 1}, {1, 1, 0}, {1, 0, 0}, {2, 1, 0}, {2, 0, 0},
      {0, 1, 2}, {0, 0, 2}, {1, 1, 2}, {1, 0, 2}, {2, 1, 1}, {2, 0, 1}};
  const int(*passes)[3] = is_e ? e_passes : h_passes;
  for (int p = 0; p < 12; ++p) {
    tfsf_pass(y, t, step, passes[p][0], passes[p][1], is_e, passes[p][2]);
  }
}

/* ------------------------------------------------------------------------
 * Lumped current / voltage source: CurrentSourceCorrector::correctE and
 * VoltageSourceCorrector::correctE
 * (src/object/lumped_element/lumped_element_corrrector.cpp:8-37):
 *   E_box += coff * waveform[t]
 * Lumped inductor (j != NULL): InductorCorrector::correctE (same file,
 * 42-99), per node in i, j, k order:
 *   E += cecjc * J;  J += cjcec * E        (cjcec in coff)
 * ---------------------------------------------------------------------- */
typedef struct {
  int comp;
  idx_t s[3], e[3];
  const double *coff;   /* box-shaped; the inductor's cjcec */
  const double *wave;   /* length nt; NULL for an inductor */
  const double *cecjc;  /* inductor: box-shaped */
  double *j;            /* inductor: box-shaped current state */
} orc_lumped;

void orc_current_source(const orc_yee *y, const orc_lumped *l, idx_t step) {
  orc_arr F = y->e[l->comp];
  const idx_t n1 = l->e[1] - l->s[1], n2 = l->e[2] - l->s[2];
  const double w = l->j ? 0.0 : l->wave[step];
  for (idx_t i = l->s[0]; i < l->e[0]; ++i)
    for (idx_t j = l->s[1]; j < l->e[1]; ++j)
      for (idx_t k = l->s[2]; k < l->e[2]; ++k) {
        const idx_t q = ((i - l->s[0]) * n1 + (j - l->s[1])) * n2 + (k - l->s[2]);
        if (l->j) {
          AT(F, i, j, k) += l->cecjc[q] * l->j[q];
          l->j[q] += l->coff[q] * AT(F, i, j, k);
        } else {
          AT(F, i, j, k) += l->coff[q] * w;
        }
      }
}

/* ------------------------------------------------------------------------
 * NF2FF frequency-domain running DFT.  NFFFTFrequencyDomain::update
 * (src/nffft/nffft_frequency_domain.cpp:45-53) loops over the frequencies
 * and, inside, over every per-frequency plane data, so each plane is
 * accumulated nF times per step; FDPlaneData::update/calculateJ/calculateM
 * (src/nffft/nffft_fd_data_update.cpp:6-122) with interpolateSurfaceCenter
 * (src/include/nffft/interpolate_scheme.h:19-138) and the phasors of
 * FDPlaneData::initDFT (src/nffft/nffft_fd_data.cpp:65-76).
 * Accumulators: per frequency f, face d (XN XP YN YP ZN ZP) and quantity
 * q (ja, jb, ma, mb) a complex array over the face task, interleaved re/im,
 * at acc + 2*off[(f*6 + d)*4 + q].
 * ---------------------------------------------------------------------- */
typedef struct {
  idx_t nf, nt;
  idx_t task_s[6][3], task_e[6][3];
  const double *te, *th;   /* (nf, nt, 2) */
  double *acc;
  const idx_t *off;
} orc_nf2ff;

static double interp_surface(const orc_yee *y, int m, int is_e, int comp, idx_t i, idx_t j,
                             idx_t k) {
  if (is_e) {
    /* 2-point averages: E_comp on face normal m averages along the third axis. */
    const orc_arr E = y->e[comp];
    idx_t q[3] = {i, j, k};
    const int other = 3 - m - comp;
    q[other] += 1;
    return 0.5 * (AT(E, q[0], q[1], q[2]) + AT(E, i, j, k));
  }
  const orc_arr H = y->h[comp];
  const int other = 3 - m - comp;
  (void)other;
  if (m == 0) {
    /* interpolateHyFaceX / interpolateHzFaceX: step along the component axis. */
    idx_t p1[3] = {i, j, k};
    p1[comp] += 1;
    return 0.25 * (AT(H, p1[0], p1[1], p1[2]) + AT(H, i, j, k) +
                   AT(H, p1[0] - 1, p1[1], p1[2]) + AT(H, i - 1, j, k));
  }
  if (m == 1) {
    if (comp == 2) { /* interpolateHzFaceY */
      return 0.25 * (AT(H, i, j, k + 1) + AT(H, i, j, k) + AT(H, i, j - 1, k + 1) +
                     +AT(H, i, j - 1, k));
    }
    /* interpolateHxFaceY */
    return 0.25 * (AT(H, i + 1, j, k) + AT(H, i, j, k) + AT(H, i + 1, j - 1, k) +
                   AT(H, i, j - 1, k));
  }
  if (comp == 0) { /* interpolateHxFaceZ */
    return 0.25 * (AT(H, i + 1, j, k) + AT(H, i, j, k) + AT(H, i, j, k - 1) +
                   AT(H, i + 1, j, k - 1));
  }
  /* interpolateHyFaceZ */
  return 0.25 * (AT(H, i, j, k) + AT(H, i, j + 1, k) + AT(H, i, j, k - 1) +
                 AT(H, i, j + 1, k - 1));
}

static void nf2ff_plane_update(const orc_yee *y, const orc_nf2ff *nf, idx_t f, idx_t step) {
  const double *te = nf->te + (f * nf->nt + step) * 2;
  const double *th = nf->th + (f * nf->nt + step) * 2;
  /* calculateJ for all six faces, then calculateM for all six. */
  for (int pass = 0; pass < 2; ++pass) {
    const int is_m = pass;
    for (int d = 0; d < 6; ++d) {
      const int m = d / 2;
      const int positive = d % 2;
      const idx_t *s = nf->task_s[d], *e = nf->task_e[d];
      if (e[0] <= s[0] || e[1] <= s[1] || e[2] <= s[2]) continue;
      const int A = tan_a(m), B = tan_b(m);
      const idx_t n1 = e[1] - s[1], n2 = e[2] - s[2];
      double c1, c2;
      const double *ph;
      if (!is_m) {
        c1 = positive ? -1.0 : 1.0; /* coff_ja */
        c2 = positive ? 1.0 : -1.0; /* coff_jb */
        ph = th;
      } else {
        c1 = positive ? 1.0 : -1.0; /* coff_ma */
        c2 = positive ? -1.0 : 1.0; /* coff_mb */
        ph = te;
      }
      double *acc1 = nf->acc + 2 * nf->off[((f * 6 + d) * 4) + (is_m ? 2 : 0)];
      double *acc2 = nf->acc + 2 * nf->off[((f * 6 + d) * 4) + (is_m ? 3 : 1)];
      /* Points are independent: each keeps the reference's order of additions,
       * so the threads change nothing but the time. */
#pragma omp parallel for collapse(2) schedule(static)
      for (idx_t i = s[0]; i < e[0]; ++i)
        for (idx_t j = s[1]; j < e[1]; ++j)
          for (idx_t k = s[2]; k < e[2]; ++k) {
            const idx_t q = ((i - s[0]) * n1 + (j - s[1])) * n2 + (k - s[2]);
            /* ja/ma use the B-component, jb/mb the A-component. */
            const double v1 = c1 * interp_surface(y, m, is_m, B, i, j, k);
            const double v2 = c2 * interp_surface(y, m, is_m, A, i, j, k);
            acc1[2 * q] += v1 * ph[0];
            acc1[2 * q + 1] += v1 * ph[1];
            acc2[2 * q] += v2 * ph[0];
            acc2[2 * q + 1] += v2 * ph[1];
          }
    }
  }
}

void orc_nf2ff_update(const orc_yee *y, const orc_nf2ff *nf, idx_t step) {
  for (idx_t rep = 0; rep < nf->nf; ++rep) {
    for (idx_t f = 0; f < nf->nf; ++f) {
      nf2ff_plane_update(y, nf, f, step);
    }
  }
}

/* ------------------------------------------------------------------------
 * Time-domain NF2FF: NFFFTTimeDomain::update (src/nffft/nfffft_time_domain.cpp:80-96)
 * -> TDPlaneData<D>::update<E> for the six faces, then update<H> for the six
 * (src/include/nffft/nffft_td_data.h:169-240).  Per face d: pot + (d*4 + q)*n_bins
 * holds ua, ub (q = 0, 1; from E) and wa, wb (q = 2, 3; from H) over the
 * retarded-time bins; prev holds, per point, the previous step's surface-centre
 * E_a, E_b, H_a, H_b (4 x P); delay and ds per point, faces in order, k fastest.
 * ---------------------------------------------------------------------- */
typedef struct {
  idx_t task_s[6][3], task_e[6][3];
  const double *delay, *ds;
  double *prev, *pot;
  idx_t P, n_bins;
} orc_nf2ff_td;

void orc_nf2ff_td_update(const orc_yee *y, const orc_nf2ff_td *td, idx_t step) {
  for (int attr = 0; attr < 2; ++attr) {
    const int is_e = attr == 0;
    const double offset = is_e ? 0.5 : 0.0;
    idx_t off = 0;
    for (int d = 0; d < 6; ++d) {
      const int m = d / 2;
      const int positive = d % 2;
      const idx_t *s = td->task_s[d], *e = td->task_e[d];
      if (e[0] <= s[0] || e[1] <= s[1] || e[2] <= s[2]) continue;
      const int A = tan_a(m), B = tan_b(m);
      double ca = is_e ? 1.0 : -1.0, cb = is_e ? -1.0 : 1.0;
      if (!positive) {
        ca *= -1.0;
        cb *= -1.0;
      }
      double *pa = td->pot + (d * 4 + (is_e ? 0 : 2)) * td->n_bins;
      double *pb = td->pot + (d * 4 + (is_e ? 1 : 3)) * td->n_bins;
      double *prev_a = td->prev + (is_e ? 0 : 2) * td->P;
      double *prev_b = td->prev + (is_e ? 1 : 3) * td->P;
      const idx_t n1 = e[1] - s[1], n2 = e[2] - s[2];
      for (idx_t i = s[0]; i < e[0]; ++i)
        for (idx_t j = s[1]; j < e[1]; ++j)
          for (idx_t k = s[2]; k < e[2]; ++k) {
            const idx_t q = off + ((i - s[0]) * n1 + (j - s[1])) * n2 + (k - s[2]);
            const double x = td->delay[q] + offset + (double)step;
            const idx_t nn = (idx_t)floor(x);
            const double f = x - (double)nn;
            const double ds = td->ds[q];
            const double a = interp_surface(y, m, is_e, A, i, j, k);
            const double b = interp_surface(y, m, is_e, B, i, j, k);
            const double da = a - prev_a[q], db = b - prev_b[q];
            pa[nn] += ca * (1 - f) * ds * db;
            pa[nn + 1] += ca * f * ds * db;
            pb[nn] += cb * (1 - f) * ds * da;
            pb[nn + 1] += cb * f * ds * da;
            prev_a[q] = a;
            prev_b[q] = b;
          }
      off += (e[0] - s[0]) * n1 * n2;
    }
  }
}

/* ------------------------------------------------------------------------
 * One whole time step in the order of Domain::run (src/domain/domain.cpp:82-135):
 * updateH -> correctH (objects -> TFSF -> PML slabs in insertion order)
 * -> updateE -> correctE (same corrector order) -> record (NF2FF; monitors are
 * copied by the caller).
 * ---------------------------------------------------------------------- */
typedef struct {
  orc_yee *yee;
  const orc_ade *ade;          /* NULL: BasicUpdator3D */
  const orc_pml *pml;
  idx_t n_pml;
  const orc_tfsf *tfsf;        /* NULL: none */
  const orc_lumped *lumped;
  idx_t n_lumped;
  const orc_nf2ff *nf2ff;      /* NULL: none */
  const orc_nf2ff_td *nf2ff_td;  /* NULL: none */
} orc_sim;

void orc_step(const orc_sim *s, idx_t step) {
  orc_update_h(s->yee);
  if (s->tfsf) orc_tfsf_correct(s->yee, s->tfsf, step, 0);
  for (idx_t p = 0; p < s->n_pml; ++p) orc_pml_correct(s->yee, &s->pml[p], 0);
  if (s->ade) {
    orc_update_e_ade(s->yee, s->ade);
  } else {
    orc_update_e(s->yee);
  }
  for (idx_t l = 0; l < s->n_lumped; ++l) orc_current_source(s->yee, &s->lumped[l], step);
  if (s->tfsf) orc_tfsf_correct(s->yee, s->tfsf, step, 1);
  for (idx_t p = 0; p < s->n_pml; ++p) orc_pml_correct(s->yee, &s->pml[p], 1);
  if (s->nf2ff) orc_nf2ff_update(s->yee, s->nf2ff, step);
  if (s->nf2ff_td) orc_nf2ff_td_update(s->yee, s->nf2ff_td, step);
}

void orc_run(const orc_sim *s, idx_t step0, idx_t nsteps) {
  for (idx_t t = step0; t < step0 + nsteps; ++t) orc_step(s, t);
}
