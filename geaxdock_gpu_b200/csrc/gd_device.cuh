/*
 * gd_device.cuh -- device-resident data layout of the B200 Monte Carlo docking engine.
 *
 * HBM layout (one context, all complexes of a batch):
 *   ligand conformers   float4 (x, y, z, charge) + int2 (type, MCS field) per atom,
 *                       conformer-major; placed coordinates never touch HBM.
 *   protein conformers  two copies of every conformer's points:
 *                       (1) for the all-pairs loop (vdw, ele, pmf, hdb), sorted by point type,
 *                       every type segment starting on an even slot, stored as pairs of slots
 *                       in two float4 streams (negated coordinates and ele / el1) so one
 *                       16-byte shared load gives the two-lane register pairs of the FP32x2
 *                       loop; a segment table (start, end, type, flags) per conformer, flag
 *                       bit 2: the type has a live hydrogen-bond pair with the ligand;
 *                       (2) for the short-range terms (contacts, psp, hpc, the electrostatic
 *                       soft core), a cell list: points sorted by cell of a uniform grid (x
 *                       fastest) as float4 (x, y, z, type and kind bits) + float4 (hpp, PSP
 *                       column bits, ele / el1, 0), and the first point of every cell.
 *   pair parameters     per (ligand type, protein type) 12 floats, folded for the kernel.
 *   contact reference   per conformer and ligand atom, the list of reference contacts as
 *                       float4 (x, y, z, contact threshold): tp is counted over this sparse
 *                       list, so the pair loop only counts contacts.
 *   replica state       movematrix_old[6], Energy (48 B), Replica (16 B), counters; records
 *                       in the reference's LigRecordSingleStep layout.
 * Protein tiles are staged from HBM/L2 into shared memory with cp.async.bulk (TMA engine)
 * into a double buffer completed on mbarriers.
 */
#ifndef GD_DEVICE_CUH
#define GD_DEVICE_CUH

#include <cstdint>

#include "../../include/geauxdock_b200.h"

#define GD_MAX_SEG 32          /* point types (30), rounded up */
#define GD_FAR_BINS 64         /* radius bins of the far-point counts (GdDevComplex.far_cnt) */
#define GD_CELL 4.0f           /* edge of the short-range cell grid (A) */
/* shared-memory bytes of the contact-threshold table at the front of the kernel's buffer */
#define GD_THR_BYTES (GD_MAXTP2 * GD_MAXTP1 * 4)
#define GD_MAX_CELLS (1 << 22) /* cells per conformer grid; a larger box widens the cells */
#define GD_MAX_CELLS_ALL (1 << 25) /* cells of all conformers of a complex together */
#define GD_MAX_TPB 256         /* threads per CTA: 3 CTAs of 256 fit the register file */
#define GD_SLOT_BYTES 192      /* shared-memory bytes per replica slot (sizeof gd::Slot) */
/* resident 256-thread CTAs per SM the register budget is set for, per unroll depth: 80
 * registers at four point pairs in flight, 64 below (no spills); the delayed-acceptance
 * variants keep one CTA fewer (80 at two pairs, 128 at four), where 64 and 80 would spill */
#define GD_MIN_BLOCKS(u) ((u) >= 4 ? 3 : 4)
#define GD_MIN_BLOCKS_DA(u) ((u) >= 4 ? 2 : ((u) >= 2 ? 3 : 4))
/* two replicas per thread: CTAs of at most GD_MAX_TPB / 2 threads (the tile's lanes over two),
 * 4 resident per SM with one point pair in flight per replica, 3 with two */
#define GD_MIN_BLOCKS_PACK(u, p, da) \
  ((p) == 2 ? ((u) >= 2 ? 3 : 4) : ((da) ? GD_MIN_BLOCKS_DA(u) : GD_MIN_BLOCKS(u)))
#define GD_MAX_SLOTS 128       /* replicas per CTA */
#define GD_NQ 12               /* per-lane partial sums handed to the reducer */

/* device error word bits */
#define GD_DEV_ERR_TIMEOUT 1
#define GD_DEV_ERR_RECORD_FULL 2
#define GD_DEV_ERR_CONFIG 4

struct GdPairParam {
  float p1a, p2a, p1l, thr;    /* LJ numerators; p1a*lj0; contact threshold on d^2 */
  float pmf0, pmf1, hc1, hc0;  /* pmf; hdb argument h = r*hc1 + hc0 (scaled for exp2) */
  float hs, hneed, b2, c2;     /* hdb scale (0 when hdb0 <= 0.1); 1 if the hdb term is live;
                                  pmf exponent cA d2 + b2 r + c2 in base 2 */
};

struct GdDevComplex {
  int n_lig, n_prt, n_tmp, lna;
  int pnp, pnp_pad, pnk, pos;
  int rep_offset, n_rep, psp_ld, mcs_ld;
  int stream, nref_total, pad0, pad1;
  float pocket[4];
  /* short-range cell grid, one frame for every conformer of the complex: cell (ix, iy, iz)
   * covers [org + i * cell, org + (i + 1) * cell) per axis, index (iz * ny + iy) * nx + ix */
  float sr_org[3], sr_cell, sr_inv_cell;
  float sr_r;                 /* search radius: every pair with d^2 <= sr_r2 lies inside it */
  float sr_r2;                /* max(81 (hpc), largest contact threshold, (1 / el1)^2) */
  float sr_pad;
  int sr_n[4];                /* nx, ny, nz, cells */
  const float4 *lig_pos;      /* [n_lig*lna] */
  const int2 *lig_meta;       /* [n_lig*lna] type, MCS index (n + 1) */
  const float *lig_center;    /* [n_lig*3] */
  /* protein points in pairs (slots 2m, 2m+1), [n_prt*pnp_pad/2] each:
   *   pt_a = (-x0, -x1, -y0, -y1), pt_b = (-z0, -z1, ele0 / el1, ele1 / el1) */
  const float4 *pt_a;
  const float4 *pt_b;
  /* the cell list, [n_prt*pnp] points and [n_prt*(sr_n[3] + 1)] cell starts (conformer-local
   * point indices): sr_a = (x, y, z, bits of type | 256 if hydrophobic | 512 if class 2),
   * sr_b = (hpp, PSP column bits, ele / el1, 0) */
  const float4 *sr_a;
  const float4 *sr_b;
  const int *sr_start;
  const int4 *seg;            /* [n_prt*GD_MAX_SEG] */
  const int *seg_count;       /* [n_prt] */
  const float4 *kde;          /* [pnk] x, y, z, type (exact small integer as float) */
  const float *mcs_x, *mcs_y, *mcs_z; /* [pos*mcs_ld] */
  const float *mcs_tcc;       /* [pos] */
  const float *psp;           /* [GD_MAXTP2*psp_ld] */
  const float *minus_beta;    /* [n_tmp] */
  const int *ref_start;       /* [n_prt*(lna+1)] */
  const float4 *ref_pts;      /* [ref_start[n_prt*(lna+1)-1]] */
  /* Within each segment the points run by distance from the pocket centre. far_cnt[(pc *
   * GD_MAX_SEG + seg) * GD_FAR_BINS + b]: how many of the segment's points lie closer than
   * (b + 1) / far_inv_w to the centre (all of them at the last bin). A point further than
   * far_r + (an atom's distance from the centre) from the centre is further than far_r from
   * the atom, where every type pair's pmf exponent is below -25.5 in base 2. */
  const unsigned short *far_cnt;
  float far_r, far_inv_w;
};

/* One CTA's unit of work: `count` consecutive replicas of one protein conformer. */
struct GdTileDesc {
  int complex_index, prt_conf, rep_begin, count;  /* rep_begin: global replica index */
};

struct GdForceConst {
  float lj1, el0, el1, a1, b1, inv_el1;
  float near2;                /* (1 / el1)^2: soft-core electrostatics inside */
  float kde2, kde3;
  float a_para[GD_MAXWEI], b_para[GD_MAXWEI], w[GD_MAXWEI];
  float hpl0[GD_MAXTP2], hpl1[GD_MAXTP2], hpl2[GD_MAXTP2];
};

/* Delayed-acceptance state read by the exact kernel in mode 3 (device-resident). Survivors of
 * the surrogate stage are compacted per (complex, protein conformer) group into pose slots
 * [group_b0[g], group_b0[g] + count[g]); pose_rep maps a slot to its replica. */
struct GdDaEpi {
  const int *group_b0;        /* [n_groups] */
  int n_groups, n_rep;
  const int *pose_rep;        /* [n_rep] */
  const float *s_new;         /* [n_rep] surrogate energy of the proposal */
  float *s_cur;               /* [n_rep] surrogate energy of the current pose */
  const float *u2;            /* [n_rep] final accept uniform (the plain step's) */
  const int *active;          /* [n_complex] surrogate stage on */
  int *acc, *plain_acc;       /* [n_rep] accepted moves with the stage on / off */
  double *err2;               /* [n_rep] sum of (S_new - E_new)^2 with the stage on */
  int *nerr;                  /* [n_rep] its count */
  float *smp_t;               /* [smp_cap] training targets (collect steps) */
  long long smp_cap;
  float *tr_s, *tr_e;         /* decision trace, [n_rep*tr_cap] or null */
  int *tr_flag;
  int tr_cap, tr_step0;
};

/* Arguments of the fused Monte Carlo / energy kernel. */
struct GdMcArgs {
  const GdDevComplex *cx;     /* [n_complex] */
  const GdPairParam *pp;      /* [GD_MAXTP2*GD_MAXTP1] */
  const GdTileDesc *tiles;    /* [n_tiles] */
  int n_tiles;
  int *tile_counter;          /* persistent-CTA work queue head */
  int mode;                   /* 0: MC steps, 1: init (energy at movematrix 0), 2: eval poses,
                                 3: delayed-acceptance exact stage (eval + decision), 4: eval
                                 given placed coordinates */
  int n_steps;                /* steps in this launch (mode 0) */
  int step0;                  /* step number of the first step (s1 + s2), added to *step_base */
  const int *step_base;       /* device cursor for graph replays (null: 0) */
  int chunk;                  /* protein points per shared-memory buffer (multiple of 4) */
  int split;                  /* lanes per ligand atom (protein split), >= 1 */
  int move_kind;
  uint64_t seed;
  float move_scale[6];
  /* replica state, global replica index */
  gd_replica *replica;
  float *mm_old;              /* [n_rep*6] */
  gd_energy *e_old;
  float *etotal;
  int *n_accept;
  /* records */
  gd_record_step *rec;        /* [n_rep*rec_cap] or null */
  int *rec_next;              /* [n_rep] */
  int rec_cap;
  /* trace (replay) */
  float *trace_e;             /* [n_rep*trace_cap] or null */
  int *trace_acc;
  int trace_cap, trace_step0;
  /* pose evaluation (mode 2): pose i of the tile uses mm_in[(rep_begin - 0 + j)*6] */
  const float *mm_in;
  const int *lig_conf_in;     /* per pose ligand conformer (mode 2) */
  gd_energy *e_out;
  /* mode 4: pose i's atoms at xyz_in[(i * lna + atom) * 3 + {0,1,2}], its centre at
   * center_in[i * 3 + {0,1,2}] (the lab frame, as Ligand.coord_new) */
  const float *xyz_in;
  const float *center_in;
  unsigned *err;              /* device error word */
  long long timeout_ns;       /* bounded waits */
  /* mode 3: tile.count holds (group << 8) | capacity; the survivors come from da_cnt */
  const GdDaEpi *da;
  const int *da_cnt;          /* [n_groups] survivors this step */
  int *da_cnt_next;           /* [n_groups] the next step's counters; block 0 zeroes the
                                 range [da_g0, da_g1) this launch serves */
  int da_g0, da_g1;
  int da_collect;             /* collect step: stage off everywhere, targets stored */
  /* ExchangeReplicas_d fused into mode 0 (launches that cover whole groups and one exchange
   * interval): per-group counts of replicas written back in this launch, the complexes' first
   * group, the exchange counters, and the exchange call (*x_call_base + x_call_off); mode_t
   * = !(((s mod x_spd) / x_spe) % 2) for the interval starting at step s, as the reference's
   * launcher derives it from the step within the dump window */
  int *x_done;                /* [n_groups] zeroed before the launch, or null */
  const int *x_group_base;    /* [n_complex] */
  int *x_acs;                 /* [n_rep] */
  const int *x_call_base;
  int x_call_off, x_spd, x_spe;
};

#endif
