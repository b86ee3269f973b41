/*
 * gd_oracle.c -- CPU restatement of the GeauxDock Monte Carlo path (see gd_oracle.h for
 * the reference file:line map). TEST INFRASTRUCTURE ONLY: the checker and the timed CPU
 * baseline; never linked into the product.
 */
#include "gd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The RNG stream and the decision arithmetic are the specification shared with the
 * device (counter layout, uniform conversion, exp used by the Metropolis test). */
#include "../geaxdock_gpu_b200/csrc/gd_numerics.h"

#define GDO_PI 3.1415926535f /* reference src/size.h:67 */

/* ---------------- energy, two precisions ---------------- */
#define REAL double
#define SQRT sqrt
#define EXP exp
#define LOG log
#define FABS fabs
#define ENERGY_FN gdo_energy_f64
#include "gd_oracle_energy.inc"
#undef REAL
#undef SQRT
#undef EXP
#undef LOG
#undef FABS
#undef ENERGY_FN

#define REAL float
#define SQRT sqrtf
#define EXP expf
#define LOG logf
#define FABS fabsf
#define ENERGY_FN gdo_energy_f32
#include "gd_oracle_energy.inc"
#undef REAL
#undef SQRT
#undef EXP
#undef LOG
#undef FABS
#undef ENERGY_FN

float gdo_contact_threshold(float pmf0) {
  if (!(pmf0 >= 0.0f)) return -1.0f;
  float t = (float)((double)pmf0 * (double)pmf0);
  while (t > 0.0f && sqrtf(t) > pmf0) t = nextafterf(t, -INFINITY);
  while (sqrtf(nextafterf(t, INFINITY)) <= pmf0) t = nextafterf(t, INFINITY);
  return t;
}

static void thresholds(const gd_enepara *ff, float *thr) {
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j)
      thr[i * GD_MAXTP1 + j] = gdo_contact_threshold(ff->pmf0[i][j]);
}

int gdo_energy_eval(const gd_enepara *ff, const gd_complex_desc *cx, int prt_conf,
                    int lig_conf, const float *x, const float *y, const float *z,
                    const float center[3], const uint8_t *refmap, int precision,
                    gdo_energy *out) {
  float thr[GD_MAXTP2 * GD_MAXTP1];
  thresholds(ff, thr);
  memset(out, 0, sizeof(*out));
  if (precision == 32)
    return gdo_energy_f32(ff, cx, prt_conf, lig_conf, x, y, z, center, refmap, thr, out);
  return gdo_energy_f64(ff, cx, prt_conf, lig_conf, x, y, z, center, refmap, thr, out);
}

/* ---------------- placement ---------------- */
void gdo_place_f32(const gd_complex_desc *cx, int lig_conf, const float mm[6], float *x,
                   float *y, float *z, float center[3]) {
  float rot[9];
  gd_rotation(mm, rot);
  const int L = cx->lna, lo = lig_conf * L;
  const float tx = mm[0] + cx->lig_center[lig_conf * 3 + 0];
  const float ty = mm[1] + cx->lig_center[lig_conf * 3 + 1];
  const float tz = mm[2] + cx->lig_center[lig_conf * 3 + 2];
  for (int l = 0; l < L; ++l)
    gd_place_atom(rot, tx, ty, tz, cx->lig_x[lo + l], cx->lig_y[lo + l], cx->lig_z[lo + l],
                  &x[l], &y[l], &z[l]);
  center[0] = tx;
  center[1] = ty;
  center[2] = tz;
}

void gdo_place_f64(const gd_complex_desc *cx, int lig_conf, const float mm[6], double *x,
                   double *y, double *z, double center[3]) {
  const double s1 = sin(mm[3]), c1 = cos(mm[3]);
  const double s2 = sin(mm[4]), c2 = cos(mm[4]);
  const double s3 = sin(mm[5]), c3 = cos(mm[5]);
  double rot[3][3];
  rot[0][0] = c1 * c2;
  rot[0][1] = c1 * s2 * s3 - c3 * s1;
  rot[0][2] = s1 * s3 + c1 * c3 * s2;
  rot[1][0] = c2 * s1;
  rot[1][1] = c1 * c3 + s1 * s2 * s3;
  rot[1][2] = c3 * s1 * s2 - c1 * s3;
  rot[2][0] = -s2;
  rot[2][1] = c2 * s3;
  rot[2][2] = c2 * c3;
  const int L = cx->lna, lo = lig_conf * L;
  const double cxx = cx->lig_center[lig_conf * 3 + 0];
  const double cyy = cx->lig_center[lig_conf * 3 + 1];
  const double czz = cx->lig_center[lig_conf * 3 + 2];
  for (int l = 0; l < L; ++l) {
    const double a = cx->lig_x[lo + l], b = cx->lig_y[lo + l], c = cx->lig_z[lo + l];
    x[l] = rot[0][0] * a + rot[0][1] * b + rot[0][2] * c + mm[0] + cxx;
    y[l] = rot[1][0] * a + rot[1][1] * b + rot[1][2] * c + mm[1] + cyy;
    z[l] = rot[2][0] * a + rot[2][1] * b + rot[2][2] * c + mm[2] + czz;
  }
  center[0] = cxx + mm[0];
  center[1] = cyy + mm[1];
  center[2] = czz + mm[2];
}

void gdo_ref_map(const gd_enepara *ff, const gd_complex_desc *cx, uint8_t *refmap) {
  float thr[GD_MAXTP2 * GD_MAXTP1];
  thresholds(ff, thr);
  const int L = cx->lna, P = cx->pnp;
  float *x = (float *)malloc(sizeof(float) * L * 3);
  float c[3];
  const float mm0[6] = {0, 0, 0, 0, 0, 0};
  gdo_place_f32(cx, 0, mm0, x, x + L, x + 2 * L, c);
  for (int l = 0; l < L; ++l) {
    const int tl = cx->lig_t[l];
    for (int p = 0; p < P; ++p) {
      const float dx = x[l] - cx->prt_x[p];
      const float dy = x[L + l] - cx->prt_y[p];
      const float dz = x[2 * L + l] - cx->prt_z[p];
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      refmap[(size_t)l * P + p] = d2 <= thr[tl * GD_MAXTP1 + cx->prt_t[p]];
    }
  }
  free(x);
}

/* ---------------- host folds ---------------- */
void gdo_fold_enepara(const gd_enepara_raw *raw, gd_enepara *o) {
  const float sqrt_2_pi = sqrtf(2.0f * GDO_PI);
  memset(o, 0, sizeof(*o));
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      const float tmp = raw->vdw[j][i][0] * raw->lj[2];
      o->p1a[i][j] = 2.0f * raw->vdw[j][i][1] * powf(tmp, 9.0f);
      o->p2a[i][j] = 3.0f * raw->vdw[j][i][1] * powf(tmp, 6.0f);
    }
  o->lj0 = raw->lj[0];
  o->lj1 = raw->lj[1];
  o->el0 = raw->el[0];
  o->a1 = 4.0f - 3.0f * raw->el[0];
  o->b1 = 2.0f * raw->el[0] - 3.0f;
  o->el1 = raw->el[1];
  for (int i = 0; i < GD_MAXTP3; ++i) o->ele[i] = raw->ele[i];
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      o->pmf0[i][j] = raw->pmf[j][i][0];
      o->pmf1[i][j] = raw->pmf[j][i][1];
      o->hdb0[i][j] = raw->hdb[j][i][0];
      o->hdb1[i][j] = 1.0f / raw->hdb[j][i][1];
    }
  for (int i = 0; i < GD_MAXTP4; ++i) o->hpp[i] = raw->hpp[i];
  for (int i = 0; i < GD_MAXTP2; ++i) {
    o->hpl0[i] = raw->hpl[i][0];
    o->hpl1[i] = raw->hpl[i][1];
    o->hpl2[i] = logf(1.0f / (o->hpl1[i] * sqrt_2_pi));
  }
  o->kde2 = -0.5f / (raw->kde * raw->kde);
  o->kde3 = powf(raw->kde * sqrt_2_pi, 3.0f);
  for (int i = 0; i < GD_MAXWEI; ++i) {
    o->w[i] = raw->w[i];
    o->a_para[i] = raw->a_para[i];
    o->b_para[i] = raw->b_para[i];
  }
}

void gdo_set_temperature(int num_temp, float floor_temp, float ceiling_temp, gd_temp *t) {
  if (num_temp == 1) {
    const float beta = 1.0f / (1.0f * floor_temp);
    t[0].t = floor_temp;
    t[0].order = 0;
    t[0].minus_beta = 0.0f - beta;
    return;
  }
  const float ratio = (float)exp(log(ceiling_temp / floor_temp) / (float)(num_temp - 1));
  float a = floor_temp;
  for (int i = 0; i < num_temp; ++i) {
    const float beta = 1.0f / (1.0f * a);
    t[i].t = a;
    t[i].order = i;
    t[i].minus_beta = 0.0f - beta;
    a *= ratio;
  }
}

/* ---------------- RNG / decision primitives ---------------- */
void gdo_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                uint32_t out[4]) {
  const gd_u32x4 r = gd_philox4x32_10(c0, c1, c2, c3, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}
float gdo_expf(float x) { return gd_expf(x); }
float gdo_logf(float x) { return gd_logf(x); }
void gdo_sincosf(float x, float *s, float *c) { gd_sincosf(x, s, c); }

void gdo_draw_steps(uint64_t seed, uint32_t stream, int move_kind, const float scale[6], int n,
                    const uint32_t *replica, const uint32_t *step, float *delta6, float *u) {
  for (int i = 0; i < n; ++i)
    gd_draw_step(seed, stream, replica[i], step[i], move_kind, scale, delta6 + 6 * i, u + i);
}

void gdo_metropolis_batch(int n, const float *e_new, const float *e_old, const float *mb,
                          const float *u, int32_t *out) {
  for (int i = 0; i < n; ++i) out[i] = gd_metropolis(e_new[i], e_old[i], mb[i], u[i]);
}

float gdo_draw_exchange(uint64_t seed, uint32_t stream, uint32_t group, uint32_t call,
                        uint32_t pair) {
  return gd_draw_exchange(seed, stream, group, call, pair);
}

int gdo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---------------- Monte Carlo chain set ---------------- */
struct gdo_mc {
  gd_enepara ff;
  gd_complex_desc cx;
  gd_mc_params mc;
  int stream, n_rep, cap, precision, n_exchange_calls;
  gd_replica *replica;
  float *mm_old;
  gd_energy *e_old;
  float *etotal;
  int32_t *n_accept, *acs;
  gd_record_step *rec;
  int32_t *next_ptr;
  uint8_t *refmap;
  float thr[GD_MAXTP2 * GD_MAXTP1];
};

gdo_mc *gdo_mc_create(const gd_enepara *ff, const gd_complex_desc *cx, const gd_mc_params *mc,
                      int stream, int precision) {
  gdo_mc *m = (gdo_mc *)calloc(1, sizeof(gdo_mc));
  m->ff = *ff;
  m->cx = *cx;
  m->mc = *mc;
  m->stream = stream;
  m->precision = precision;
  m->n_rep = cx->n_prt * cx->n_tmp * cx->n_lig;
  m->cap = mc->steps_per_dump + 1;
  m->replica = (gd_replica *)calloc(m->n_rep, sizeof(gd_replica));
  m->mm_old = (float *)calloc((size_t)m->n_rep * 6, sizeof(float));
  m->e_old = (gd_energy *)calloc(m->n_rep, sizeof(gd_energy));
  m->etotal = (float *)calloc(m->n_rep, sizeof(float));
  m->n_accept = (int32_t *)calloc(m->n_rep, sizeof(int32_t));
  m->acs = (int32_t *)calloc(m->n_rep, sizeof(int32_t));
  m->next_ptr = (int32_t *)calloc(m->n_rep, sizeof(int32_t));
  if (mc->record)
    m->rec = (gd_record_step *)calloc((size_t)m->n_rep * m->cap, sizeof(gd_record_step));
  m->refmap = (uint8_t *)calloc((size_t)cx->lna * cx->pnp, 1);
  thresholds(ff, m->thr);
  /* SetReplica (src/util.C:842-861) */
  for (int p = 0; p < cx->n_prt; ++p)
    for (int t = 0; t < cx->n_tmp; ++t)
      for (int l = 0; l < cx->n_lig; ++l) {
        const int f = cx->n_tmp * cx->n_lig * p + cx->n_lig * t + l;
        m->replica[f].idx_rep = f;
        m->replica[f].idx_prt = p;
        m->replica[f].idx_tmp = t;
        m->replica[f].idx_lig = l;
      }
  return m;
}

void gdo_mc_destroy(gdo_mc *m) {
  if (!m) return;
  free(m->replica);
  free(m->mm_old);
  free(m->e_old);
  free(m->etotal);
  free(m->n_accept);
  free(m->acs);
  free(m->next_ptr);
  free(m->rec);
  free(m->refmap);
  free(m);
}

int gdo_mc_num_replicas(const gdo_mc *m) { return m->n_rep; }

static void to_energy(const gdo_energy *o, gd_energy *e) {
  for (int i = 0; i < GD_MAXWEI; ++i) e->e[i] = (float)o->e[i];
  e->cms = (float)o->cms;
  e->rmsd = (float)o->rmsd;
}

static void eval_pose(const gdo_mc *m, int r, const float mm[6], gd_energy *e) {
  const int L = m->cx.lna;
  float buf[3 * GD_MAXLIG], c[3];
  const int il = m->replica[r].idx_lig, ip = m->replica[r].idx_prt;
  gdo_place_f32(&m->cx, il, mm, buf, buf + L, buf + 2 * L, c);
  gdo_energy o;
  memset(&o, 0, sizeof(o));
  if (m->precision == 32)
    gdo_energy_f32(&m->ff, &m->cx, ip, il, buf, buf + L, buf + 2 * L, c, m->refmap, m->thr, &o);
  else
    gdo_energy_f64(&m->ff, &m->cx, ip, il, buf, buf + L, buf + 2 * L, c, m->refmap, m->thr, &o);
  to_energy(&o, e);
}

static void record(gdo_mc *m, int r, int step) {
  if (!m->rec) return;
  const int k = m->next_ptr[r];
  if (k >= m->cap) return; /* overflow: the device reports GD_ERR_RECORD_FULL */
  gd_record_step *s = &m->rec[(size_t)r * m->cap + k];
  s->replica = m->replica[r];
  s->energy = m->e_old[r];
  for (int i = 0; i < 6; ++i) s->movematrix[i] = m->mm_old[r * 6 + i];
  s->step = step;
  m->next_ptr[r] = k + 1;
}

void gdo_mc_init(gdo_mc *m) {
  gdo_ref_map(&m->ff, &m->cx, m->refmap);
  const float mm0[6] = {0, 0, 0, 0, 0, 0};
  for (int r = 0; r < m->n_rep; ++r) {
    for (int i = 0; i < 6; ++i) m->mm_old[r * 6 + i] = 0.0f;
    eval_pose(m, r, mm0, &m->e_old[r]);
    m->etotal[r] = m->e_old[r].e[GD_MAXWEI - 1];
    m->next_ptr[r] = 0;
    m->acs[r] = 0;
    m->n_accept[r] = 0;
    record(m, r, 0);
  }
  m->n_exchange_calls = 0;
}

void gdo_mc_reset_records(gdo_mc *m) {
  for (int r = 0; r < m->n_rep; ++r) m->next_ptr[r] = 0;
}

static void run_one(gdo_mc *m, int r, int s1, int s2, int n_steps) {
  const float mb = m->cx.temp[m->replica[r].idx_tmp].minus_beta;
  for (int s3 = 0; s3 < n_steps; ++s3) {
    const int step = s1 + s2 + s3;
    float delta[6], u, mm[6];
    gd_draw_step(m->mc.seed, (uint32_t)m->stream, (uint32_t)r, (uint32_t)step, m->mc.move_kind,
                 m->mc.move_scale, delta, &u);
    for (int i = 0; i < 6; ++i) mm[i] = GD_ADD(m->mm_old[r * 6 + i], delta[i]);
    gd_energy en;
    eval_pose(m, r, mm, &en);
    if (gd_metropolis(en.e[GD_MAXWEI - 1], m->e_old[r].e[GD_MAXWEI - 1], mb, u)) {
      for (int i = 0; i < 6; ++i) m->mm_old[r * 6 + i] = mm[i];
      m->e_old[r] = en;
      m->n_accept[r] += 1;
      record(m, r, step);
    }
  }
  m->etotal[r] = m->e_old[r].e[GD_MAXWEI - 1];
}

void gdo_mc_run_range(gdo_mc *m, int r0, int r1, int s1, int s2, int n_steps, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int r = r0; r < r1; ++r) run_one(m, r, s1, s2, n_steps);
}

void gdo_mc_run(gdo_mc *m, int s1, int s2, int n_steps, int nthreads) {
  gdo_mc_run_range(m, 0, m->n_rep, s1, s2, n_steps, nthreads);
}

void gdo_exchange_apply(const gd_complex_desc *cx, uint64_t seed, int stream,
                        int exchange_call, int mode_t, gd_replica *replica, const float *etotal,
                        int32_t *acs) {
  const int nt = cx->n_tmp, nl = cx->n_lig;
  int temps[GD_MAXTMP], orders[GD_MAXTMP];
  float en[GD_MAXTMP];
  if (mode_t >= 2) return;
  for (int p = 0; p < cx->n_prt; ++p)
    for (int l = 0; l < nl; ++l) {
      const uint32_t group = (uint32_t)(p * nl + l);
      for (int t = 0; t < nt; ++t) {
        const int f = nt * nl * p + nl * t + l;
        temps[t] = replica[f].idx_tmp;
        en[t] = etotal[f];
        orders[temps[t]] = t;
      }
      const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
      for (int pair = 0; pair < maxpair; ++pair) {
        const int i1 = (pair << 1) + mode_t, i2 = i1 + 1;
        const int o1 = orders[i1], o2 = orders[i2];
        const int tt = temps[o1];
        const float mb1 = cx->temp[temps[o1]].minus_beta;
        const float mb2 = cx->temp[temps[o2]].minus_beta;
        const float u = gd_draw_exchange(seed, (uint32_t)stream, group, (uint32_t)exchange_call,
                                         (uint32_t)pair);
        if (gd_exchange_accept(en[o1], en[o2], mb1, mb2, u)) {
          temps[o1] = temps[o2];
          temps[o2] = tt;
          if (acs) {
            acs[nt * nl * p + nl * o1 + l] += 1;
            acs[nt * nl * p + nl * o2 + l] += 1;
          }
        }
      }
      for (int t = 0; t < nt; ++t) replica[nt * nl * p + nl * t + l].idx_tmp = temps[t];
    }
}

void gdo_mc_exchange(gdo_mc *m, int mode_t) {
  gdo_exchange_apply(&m->cx, m->mc.seed, m->stream, m->n_exchange_calls, mode_t, m->replica,
                     m->etotal, m->acs);
  m->n_exchange_calls += 1;
}

int gdo_mc_exchange_calls(const gdo_mc *m) { return m->n_exchange_calls; }
void gdo_mc_set_exchange_calls(gdo_mc *m, int n) { m->n_exchange_calls = n; }

void gdo_mc_get(const gdo_mc *m, gd_replica *replica, float *mm_old, gd_energy *e_old,
                float *etotal, int32_t *n_accept, int32_t *acs) {
  const size_t n = (size_t)m->n_rep;
  if (replica) memcpy(replica, m->replica, n * sizeof(gd_replica));
  if (mm_old) memcpy(mm_old, m->mm_old, n * 6 * sizeof(float));
  if (e_old) memcpy(e_old, m->e_old, n * sizeof(gd_energy));
  if (etotal) memcpy(etotal, m->etotal, n * sizeof(float));
  if (n_accept) memcpy(n_accept, m->n_accept, n * sizeof(int32_t));
  if (acs) memcpy(acs, m->acs, n * sizeof(int32_t));
}

void gdo_mc_set(gdo_mc *m, const gd_replica *replica, const float *mm_old,
                const gd_energy *e_old, const float *etotal) {
  const size_t n = (size_t)m->n_rep;
  if (replica) memcpy(m->replica, replica, n * sizeof(gd_replica));
  if (mm_old) memcpy(m->mm_old, mm_old, n * 6 * sizeof(float));
  if (e_old) memcpy(m->e_old, e_old, n * sizeof(gd_energy));
  if (etotal) memcpy(m->etotal, etotal, n * sizeof(float));
}

int gdo_mc_get_records(const gdo_mc *m, gd_record_step *steps, int32_t *next_ptr) {
  if (!m->rec) return -1;
  memcpy(steps, m->rec, (size_t)m->n_rep * m->cap * sizeof(gd_record_step));
  memcpy(next_ptr, m->next_ptr, (size_t)m->n_rep * sizeof(int32_t));
  return m->cap;
}

const uint8_t *gdo_mc_refmap(const gdo_mc *m) { return m->refmap; }
