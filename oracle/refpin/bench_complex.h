/*
 * bench_complex.h -- a complex handed over as the product's arrays (a named-array container
 * written by oracle/refbench.py) turned into the reference's own structs (src/dock.h,
 * src/dock_soa.h) as its host preparation leaves them: Ligand / Protein / Psp / Kde / Mcs /
 * EnePara / Temp, then SetReplica and InitLigCoord (src/util.C:842-861, 439-455).
 * TEST / BENCHMARK INFRASTRUCTURE ONLY: shared by the pin harness (refpin --bench, the
 * reference's step functions on the CPU) and the GPU witness (refgpu, the reference's own Run
 * and kernels built for the GPU). Needs dock.h, size.h and util.h of the reference first.
 */
#ifndef GD_REF_BENCH_COMPLEX_H
#define GD_REF_BENCH_COMPLEX_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

/* ---------------- named-array container, reading side ---------------- */
struct Reader {
  std::map<std::string, std::vector<char>> data;
  std::map<std::string, std::vector<uint64_t>> dims;
  bool ok = false;
  explicit Reader(const char *path) {
    FILE *f = fopen(path, "rb");
    if (!f) return;
    char magic[6];
    if (fread(magic, 1, 6, f) != 6 || memcmp(magic, "GDFX1\n", 6)) { fclose(f); return; }
    for (;;) {
      uint32_t n;
      if (fread(&n, 4, 1, f) != 1) break;
      std::string name(n, ' ');
      if (fread(&name[0], 1, n, f) != n) break;
      char dt;
      uint32_t nd;
      if (fread(&dt, 1, 1, f) != 1 || fread(&nd, 4, 1, f) != 1) break;
      std::vector<uint64_t> d(nd);
      uint64_t count = 1;
      for (uint32_t i = 0; i < nd; ++i) {
        if (fread(&d[i], 8, 1, f) != 1) { fclose(f); return; }
        count *= d[i];
      }
      std::vector<char> buf(count * 4);
      if (fread(buf.data(), 1, buf.size(), f) != buf.size()) break;
      data[name] = buf;
      dims[name] = d;
    }
    fclose(f);
    ok = true;
  }
  const float *f(const char *n) const { return (const float *)data.at(n).data(); }
  const int *i(const char *n) const { return (const int *)data.at(n).data(); }
  uint64_t dim(const char *n, int k) const { return dims.at(n)[k]; }
};

/* The reference's structs of one complex, with n_rep Ligand copies as Run expects them. */
struct BenchComplex {
  ComplexSize cs;
  Ligand *lig = nullptr;
  Protein *prt = nullptr;
  Psp *psp = nullptr;
  Kde *kde = nullptr;
  Mcs *mcs = nullptr;
  EnePara *ep = nullptr;
  Temp *temp = nullptr;
  Replica *replica = nullptr;
  float move_scale[6];
  int move_kind = 0;
};

/* false when the container cannot be read or a size exceeds the reference's capacities */
static bool read_bench_complex(const Reader &rd, BenchComplex *b) {
  if (!rd.ok) return false;
  const int *sz = rd.i("sizes");
  ComplexSize &cs = b->cs;
  cs.n_lig = sz[0]; cs.n_prt = sz[1]; cs.n_tmp = sz[2]; cs.lna = sz[3]; cs.pnp = sz[4];
  cs.pnk = sz[5]; cs.pos = sz[6];
  cs.n_rep = cs.n_lig * cs.n_prt * cs.n_tmp;
  if (cs.lna > MAXLIG || cs.pnp > MAXPRO || cs.pnk > MAXKDE || cs.pos > MAXPOS) return false;
  b->move_kind = rd.data.count("move_kind") ? rd.i("move_kind")[0] : 0;
  const float *ms = rd.f("move_scale");
  for (int k = 0; k < 6; ++k) b->move_scale[k] = ms[k];
  const int L = cs.lna, P = cs.pnp;
  Ligand *lig = b->lig = (Ligand *)calloc(cs.n_rep, sizeof(Ligand));
  Protein *prt = b->prt = (Protein *)calloc(cs.n_prt, sizeof(Protein));
  Psp *psp = b->psp = (Psp *)calloc(1, sizeof(Psp));
  Kde *kde = b->kde = (Kde *)calloc(1, sizeof(Kde));
  Mcs *mcs = b->mcs = (Mcs *)calloc(cs.pos, sizeof(Mcs));
  b->ep = (EnePara *)calloc(1, sizeof(EnePara));
  b->temp = (Temp *)calloc(cs.n_tmp, sizeof(Temp));
  b->replica = (Replica *)calloc(cs.n_rep, sizeof(Replica));
  for (int c = 0; c < cs.n_lig; ++c) {
    for (int a = 0; a < L; ++a) {
      lig[c].coord_orig.x[a] = rd.f("lig_x")[c * L + a];
      lig[c].coord_orig.y[a] = rd.f("lig_y")[c * L + a];
      lig[c].coord_orig.z[a] = rd.f("lig_z")[c * L + a];
      lig[c].t[a] = rd.i("lig_t")[c * L + a];
      lig[c].c[a] = rd.f("lig_c")[c * L + a];
      lig[c].n[a] = rd.i("lig_n")[c * L + a];
    }
    for (int k = 0; k < 3; ++k) lig[c].coord_orig.center[k] = rd.f("lig_center")[c * 3 + k];
    lig[c].lna = L;
  }
  for (int c = 0; c < cs.n_prt; ++c) {
    for (int q = 0; q < P; ++q) {
      prt[c].x[q] = rd.f("prt_x")[c * P + q];
      prt[c].y[q] = rd.f("prt_y")[c * P + q];
      prt[c].z[q] = rd.f("prt_z")[c * P + q];
      prt[c].t[q] = rd.i("prt_t")[c * P + q];
      prt[c].c[q] = rd.i("prt_c")[c * P + q];
      prt[c].ele[q] = rd.f("prt_ele")[c * P + q];
      prt[c].seq3r[q] = rd.i("prt_seq3r")[c * P + q];
      prt[c].c0_and_d12_or_c2[q] = rd.i("prt_hflag")[c * P + q];
      prt[c].hpp[q] = rd.f("prt_hpp")[c * P + q];
    }
    prt[c].pnp = P;
    for (int k = 0; k < 3; ++k) prt[c].pocket_center[k] = rd.f("pocket_center")[k];
  }
  {
    const uint64_t ld = rd.dim("psp", 1);
    for (int t = 0; t < MAXTP2; ++t)
      for (uint64_t j = 0; j < ld && j < MAXPRO; ++j) psp->psp[t][j] = rd.f("psp")[t * ld + j];
  }
  for (int q = 0; q < cs.pnk; ++q) {
    kde->x[q] = rd.f("kde_x")[q];
    kde->y[q] = rd.f("kde_y")[q];
    kde->z[q] = rd.f("kde_z")[q];
    kde->t[q] = rd.i("kde_t")[q];
  }
  kde->pnk = cs.pnk;
  {
    const uint64_t ld = rd.dim("mcs_x", 1);
    for (int m = 0; m < cs.pos; ++m) {
      for (int j = 0; j < MAXMCS; ++j) {
        const bool in = (uint64_t)j < ld;
        mcs[m].x[j] = in ? rd.f("mcs_x")[m * ld + j] : 728492.0f;
        mcs[m].y[j] = in ? rd.f("mcs_y")[m * ld + j] : 728492.0f;
        mcs[m].z[j] = in ? rd.f("mcs_z")[m * ld + j] : 728492.0f;
      }
      mcs[m].tcc = rd.f("mcs_tcc")[m];
    }
  }
  memcpy(b->ep, rd.f("enepara"), sizeof(EnePara));
  memcpy(b->temp, rd.f("temp"), sizeof(Temp) * cs.n_tmp);
  SetReplica(b->replica, lig, cs);
  InitLigCoord(lig, cs);
  return true;
}

#endif
