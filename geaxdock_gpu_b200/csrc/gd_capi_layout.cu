/*
 * gd_capi_layout.cu -- the device layout of one complex (gd_create): ligand conformers, the
 * protein's two copies (type segments of point pairs for the all-pairs loop, the cell list of
 * the short-range terms), the contact reference, KDE, MCS, PSP and temperatures.
 */
#include "gd_capi_internal.cuh"

namespace gdc {

int layout_complex(gd_ctx *c, const gd_enepara *ff, const float (*thr)[GD_MAXTP1],
                   const gd_complex_desc &d, int ci, GdDevComplex &g) {
  const ComplexInfo &x = c->info[ci];
  const GdForceConst &f = c->fc;
  int rc = GD_OK;
  memset(&g, 0, sizeof(g));
  g.n_lig = d.n_lig; g.n_prt = d.n_prt; g.n_tmp = d.n_tmp; g.lna = d.lna;
  g.pnp = d.pnp; g.pnp_pad = x.pnp_pad; g.pnk = d.pnk; g.pos = d.pos;
  g.rep_offset = x.rep_offset; g.n_rep = x.n_rep; g.psp_ld = d.psp_ld; g.mcs_ld = d.mcs_ld;
  g.stream = ci;
  g.pocket[0] = d.pocket_center[0];
  g.pocket[1] = d.pocket_center[1];
  g.pocket[2] = d.pocket_center[2];
  const int L = d.lna, P = d.pnp;

  std::vector<float4> lig_pos((size_t)d.n_lig * L);
  std::vector<int2> lig_meta((size_t)d.n_lig * L);
  for (int i = 0; i < d.n_lig * L; ++i) {
    lig_pos[i] = make_float4(d.lig_x[i], d.lig_y[i], d.lig_z[i], d.lig_c[i]);
    lig_meta[i] = make_int2(d.lig_t[i], d.lig_n[i] + 1);
  }
  std::vector<float> lig_center(d.lig_center, d.lig_center + 3 * d.n_lig);
  std::vector<float4> sr_a, sr_b;
  std::vector<int> sr_start;

  /* protein, all-pairs copy: sort by point type into segments that start on even slots (one
   * padding slot after an odd-length segment), each segment by distance from the pocket
   * centre, then write slot pairs */
  std::vector<int4> seg((size_t)d.n_prt * GD_MAX_SEG, make_int4(0, 0, 0, 0));
  std::vector<int> seg_count(d.n_prt, 0);
  std::vector<std::vector<int>> slot_point(d.n_prt); /* point index per slot, -1: padding */
  int max_slots = 4;
  /* the hydrogen-bond term runs for a point type when any atom type of this ligand has a
   * live pair with it: one decision per segment for the whole CTA */
  bool hdb_live[GD_MAXTP1] = {false};
  bool lt_used[GD_MAXTP2] = {false};
  for (int i = 0; i < d.n_lig * L; ++i) lt_used[d.lig_t[i]] = true;
  for (int tp = 0; tp < GD_MAXTP1; ++tp)
    for (int tl = 0; tl < GD_MAXTP2; ++tl)
      if (lt_used[tl] && ff->hdb0[tl][tp] > 0.1f) hdb_live[tp] = true;
  /* distance of every point from the pocket centre (the kernel's float centre) */
  std::vector<double> rad((size_t)d.n_prt * P);
  double rad_max = 0.0;
  for (size_t i = 0; i < rad.size(); ++i) {
    const double dx = (double)d.prt_x[i] - (double)g.pocket[0];
    const double dy = (double)d.prt_y[i] - (double)g.pocket[1];
    const double dz = (double)d.prt_z[i] - (double)g.pocket[2];
    rad[i] = std::sqrt(dx * dx + dy * dy + dz * dz);
    rad_max = std::max(rad_max, rad[i]);
  }
  for (int pc = 0; pc < d.n_prt; ++pc) {
    const int o = pc * P;
    std::vector<int> order(P);
    for (int p = 0; p < P; ++p) order[p] = p;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const int ta = d.prt_t[o + a], tb = d.prt_t[o + b];
      return ta != tb ? ta < tb : rad[o + a] < rad[o + b];
    });
    std::vector<int> &sp = slot_point[pc];
    int ns = 0;
    for (int i = 0; i < P; ++i) {
      const int p = order[i], tp = d.prt_t[o + p];
      if (i == 0 || tp != d.prt_t[o + order[i - 1]]) {
        if (sp.size() & 1) sp.push_back(-1);
        if (ns == GD_MAX_SEG) return fail(GD_ERR_CAPACITY, "too many point segments");
        const int s0 = (int)sp.size();
        seg[(size_t)pc * GD_MAX_SEG + ns] = make_int4(s0, s0 + 1, tp, hdb_live[tp] ? 4 : 0);
        ++ns;
      } else {
        seg[(size_t)pc * GD_MAX_SEG + ns - 1].y = (int)sp.size() + 1;
      }
      sp.push_back(p);
    }
    seg_count[pc] = ns;
    max_slots = std::max(max_slots, (int)sp.size());
  }
  /* far-point counts per (conformer, segment, radius bin), and the pmf far radius: the largest
   * pmf_far_radius of the complex's type pairs plus 0.01 A for the kernel's FP32 distances */
  const double bin_w = (rad_max + 1e-3) / (GD_FAR_BINS - 1);
  std::vector<unsigned short> far_cnt((size_t)d.n_prt * GD_MAX_SEG * GD_FAR_BINS, 0);
  for (int pc = 0; pc < d.n_prt; ++pc)
    for (int sg = 0; sg < seg_count[pc]; ++sg) {
      const int4 gs = seg[(size_t)pc * GD_MAX_SEG + sg];
      if (gs.y - gs.x > 65535) return fail(GD_ERR_CAPACITY, "point segment too long");
      unsigned short *fc = &far_cnt[((size_t)pc * GD_MAX_SEG + sg) * GD_FAR_BINS];
      int n = 0;
      for (int b = 0; b < GD_FAR_BINS; ++b) {
        const double lim = (b + 1) * bin_w;
        while (gs.x + n < gs.y && (b == GD_FAR_BINS - 1 ||
                                   rad[(size_t)pc * P + slot_point[pc][gs.x + n]] < lim))
          ++n;
        fc[b] = (unsigned short)n;
      }
    }
  {
    bool pt_used[GD_MAXTP1] = {false};
    for (int i = 0; i < d.n_prt * P; ++i) pt_used[d.prt_t[i]] = true;
    double rfar = 0.0;
    for (int tl = 0; tl < GD_MAXTP2; ++tl)
      for (int tp = 0; tp < GD_MAXTP1; ++tp)
        if (lt_used[tl] && pt_used[tp]) rfar = std::max(rfar, pmf_far_radius(ff->pmf0[tl][tp]));
    g.far_r = (float)(rfar + 0.01);
    g.far_inv_w = (float)(1.0 / bin_w);
  }
  const int PP = (max_slots + 3) & ~3;
  c->info[ci].pnp_pad = PP;
  g.pnp_pad = PP;
  const size_t npair = (size_t)PP / 2;
  const float inv_el1 = 1.0f / ff->el1;
  std::vector<float4> pt_a((size_t)d.n_prt * npair, make_float4(-1e6f, -1e6f, -1e6f, -1e6f));
  std::vector<float4> pt_b((size_t)d.n_prt * npair, make_float4(-1e6f, -1e6f, 0.0f, 0.0f));
  for (int pc = 0; pc < d.n_prt; ++pc) {
    const int o = pc * P;
    const std::vector<int> &sp = slot_point[pc];
    for (size_t sidx = 0; sidx < sp.size(); ++sidx) {
      const int p = sp[sidx];
      if (p < 0) continue;
      float *A = &pt_a[pc * npair + sidx / 2].x;
      float *B = &pt_b[pc * npair + sidx / 2].x;
      const int h = (int)(sidx & 1);
      A[0 + h] = -d.prt_x[o + p];
      A[2 + h] = -d.prt_y[o + p];
      B[0 + h] = -d.prt_z[o + p];
      B[2 + h] = d.prt_ele[o + p] * inv_el1; /* ele_p / el1 */
    }
  }

  /* protein, short-range copy: a cell list over one grid frame for every conformer. The
   * search radius covers the hpc cut-off (d^2 <= 81), the largest contact threshold of the
   * complex's type pairs and the soft-core radius 1 / el1, plus 0.05 A for the rounding of
   * the kernel's cell ranges. */
  {
    bool pt_used[GD_MAXTP1] = {false};
    for (int i = 0; i < d.n_prt * P; ++i) pt_used[d.prt_t[i]] = true;
    float r2 = std::max(81.0f, f.near2);
    for (int tl = 0; tl < GD_MAXTP2; ++tl)
      for (int tp = 0; tp < GD_MAXTP1; ++tp)
        if (lt_used[tl] && pt_used[tp]) r2 = std::max(r2, thr[tl][tp]);
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < d.n_prt * P; ++i) {
      const double v[3] = {d.prt_x[i], d.prt_y[i], d.prt_z[i]};
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], v[a]);
        hi[a] = std::max(hi[a], v[a]);
      }
    }
    double cell = GD_CELL;
    long long n[3];
    /* the cell starts of all conformers share one budget (GD_MAX_CELLS_ALL) */
    const long long max_cells =
        std::max(4096LL, std::min((long long)GD_MAX_CELLS, (long long)GD_MAX_CELLS_ALL / d.n_prt));
    for (;;) {
      for (int a = 0; a < 3; ++a) n[a] = (long long)std::floor((hi[a] - lo[a] + 1.0) / cell) + 1;
      if (n[0] * n[1] * n[2] <= max_cells) break;
      cell *= 1.25;
    }
    const int ncell = (int)(n[0] * n[1] * n[2]);
    g.sr_org[0] = (float)(lo[0] - 0.5);
    g.sr_org[1] = (float)(lo[1] - 0.5);
    g.sr_org[2] = (float)(lo[2] - 0.5);
    g.sr_cell = (float)cell;
    g.sr_inv_cell = (float)(1.0 / cell);
    g.sr_r2 = r2;
    g.sr_r = sqrtf(r2) + 0.05f;
    g.sr_n[0] = (int)n[0];
    g.sr_n[1] = (int)n[1];
    g.sr_n[2] = (int)n[2];
    g.sr_n[3] = ncell;
    sr_a.assign((size_t)d.n_prt * P, make_float4(0, 0, 0, 0));
    sr_b.assign((size_t)d.n_prt * P, make_float4(0, 0, 0, 0));
    sr_start.assign((size_t)d.n_prt * (ncell + 1), 0);
    std::vector<int> cid(P);
    for (int pc = 0; pc < d.n_prt; ++pc) {
      const int o = pc * P;
      int *st = sr_start.data() + (size_t)pc * (ncell + 1);
      for (int p = 0; p < P; ++p) {
        long long ix[3];
        const double v[3] = {d.prt_x[o + p], d.prt_y[o + p], d.prt_z[o + p]};
        for (int a = 0; a < 3; ++a)
          ix[a] = std::min(n[a] - 1, std::max(0LL, (long long)std::floor(
                                                       (v[a] - (double)g.sr_org[a]) / cell)));
        cid[p] = (int)((ix[2] * n[1] + ix[1]) * n[0] + ix[0]);
        ++st[cid[p] + 1];
      }
      for (int k = 0; k < ncell; ++k) st[k + 1] += st[k];
      std::vector<int> fill(st, st + ncell);
      for (int p = 0; p < P; ++p) {
        const int i = fill[cid[p]]++;
        const int kind = (d.prt_hflag[o + p] == 1 ? 1 : 0) | (d.prt_c[o + p] == 2 ? 2 : 0);
        sr_a[(size_t)o + i] =
            make_float4(d.prt_x[o + p], d.prt_y[o + p], d.prt_z[o + p],
                        bits_as_float(d.prt_t[o + p] | (kind & 1 ? 256 : 0) |
                                      (kind & 2 ? 512 : 0)));
        sr_b[(size_t)o + i] = make_float4((kind & 1) ? d.prt_hpp[o + p] : 0.0f,
                                          bits_as_float((kind & 2) ? d.prt_seq3r[o + p] : -1),
                                          d.prt_ele[o + p] * inv_el1, 0.0f);
      }
    }
  }
  /* contact reference from (protein 0, ligand 0) at movematrix 0 (InitRefMatrix_d) */
  std::vector<int> ref_start((size_t)d.n_prt * (L + 1));
  std::vector<float4> ref_pts;
  {
    float rot[9];
    const float mm0[6] = {0, 0, 0, 0, 0, 0};
    gd_rotation(mm0, rot);
    std::vector<float> ax(L), ay(L), az(L);
    for (int l = 0; l < L; ++l)
      gd_place_atom(rot, 0.0f + d.lig_center[0], 0.0f + d.lig_center[1],
                    0.0f + d.lig_center[2], d.lig_x[l], d.lig_y[l], d.lig_z[l], &ax[l], &ay[l],
                    &az[l]);
    std::vector<std::vector<int>> refp(L);
    int nref = 0;
    for (int l = 0; l < L; ++l) {
      const int tl = d.lig_t[l];
      for (int p = 0; p < P; ++p)
        if (host_dist2(ax[l], ay[l], az[l], d.prt_x[p], d.prt_y[p], d.prt_z[p]) <=
            thr[tl][d.prt_t[p]]) {
          refp[l].push_back(p);
          ++nref;
        }
    }
    g.nref_total = nref;
    for (int pc = 0; pc < d.n_prt; ++pc) {
      const int o = pc * P;
      for (int l = 0; l < L; ++l) {
        ref_start[(size_t)pc * (L + 1) + l] = (int)ref_pts.size();
        for (int p : refp[l])
          ref_pts.push_back(make_float4(d.prt_x[o + p], d.prt_y[o + p], d.prt_z[o + p],
                                        thr[d.lig_t[l]][d.prt_t[o + p]]));
      }
      ref_start[(size_t)pc * (L + 1) + L] = (int)ref_pts.size();
    }
  }
  std::vector<float4> kde(std::max(1, d.pnk));
  for (int i = 0; i < d.pnk; ++i)
    kde[i] = make_float4(d.kde_x[i], d.kde_y[i], d.kde_z[i], (float)d.kde_t[i]);
  const size_t nm = (size_t)d.pos * d.mcs_ld;
  std::vector<float> mx(d.mcs_x, d.mcs_x + nm), my(d.mcs_y, d.mcs_y + nm),
      mz(d.mcs_z, d.mcs_z + nm), mt(d.mcs_tcc, d.mcs_tcc + d.pos);
  std::vector<float> psp(d.psp, d.psp + (size_t)GD_MAXTP2 * d.psp_ld);
  std::vector<float> mb(d.n_tmp);
  for (int t = 0; t < d.n_tmp; ++t) mb[t] = d.temp[t].minus_beta;

  float4 *p_lig_pos; int2 *p_lig_meta; float *p_lig_center; float4 *p_pt_a, *p_pt_b;
  float4 *p_sr_a, *p_sr_b; int *p_sr_start;
  int4 *p_seg; int *p_seg_count; unsigned short *p_far_cnt; float4 *p_kde; float *p_mx, *p_my, *p_mz, *p_mt, *p_psp, *p_mb;
  int *p_ref_start; float4 *p_ref_pts;
  if ((rc = upload(c, &p_lig_pos, lig_pos)) || (rc = upload(c, &p_lig_meta, lig_meta)) ||
      (rc = upload(c, &p_lig_center, lig_center)) || (rc = upload(c, &p_pt_a, pt_a)) ||
      (rc = upload(c, &p_pt_b, pt_b)) || (rc = upload(c, &p_sr_a, sr_a)) ||
      (rc = upload(c, &p_sr_b, sr_b)) || (rc = upload(c, &p_sr_start, sr_start)) ||
      (rc = upload(c, &p_seg, seg)) || (rc = upload(c, &p_far_cnt, far_cnt)) ||
      (rc = upload(c, &p_seg_count, seg_count)) || (rc = upload(c, &p_kde, kde)) ||
      (rc = upload(c, &p_mx, mx)) || (rc = upload(c, &p_my, my)) ||
      (rc = upload(c, &p_mz, mz)) || (rc = upload(c, &p_mt, mt)) ||
      (rc = upload(c, &p_psp, psp)) || (rc = upload(c, &p_mb, mb)) ||
      (rc = upload(c, &p_ref_start, ref_start)) || (rc = upload(c, &p_ref_pts, ref_pts)))
    return rc;
  /* the host vectors die at the end of this iteration: finish the copies first */
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(GD_ERR_CUDA, "upload failed: %s", cudaGetErrorString(cudaGetLastError()));
  g.lig_pos = p_lig_pos; g.lig_meta = p_lig_meta; g.lig_center = p_lig_center;
  g.pt_a = p_pt_a; g.pt_b = p_pt_b; g.seg = p_seg; g.seg_count = p_seg_count;
  g.far_cnt = p_far_cnt;
  g.sr_a = p_sr_a; g.sr_b = p_sr_b; g.sr_start = p_sr_start;
  g.kde = p_kde; g.mcs_x = p_mx; g.mcs_y = p_my; g.mcs_z = p_mz; g.mcs_tcc = p_mt;
  g.psp = p_psp; g.minus_beta = p_mb; g.ref_start = p_ref_start; g.ref_pts = p_ref_pts;
  return GD_OK;
}

}  // namespace gdc
