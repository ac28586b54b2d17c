/*
 * hb_oracle.c -- CPU oracle for the D3Q19 collide-and-stream step.
 *
 * TEST INFRASTRUCTURE ONLY (see hb_oracle.h).  A plain-C restatement of the
 * reference's single-rank lb::LBM time step, kept in the reference's push form,
 * site order and floating-point association order so that it reproduces the
 * reference's FP64 results.  Compile with -ffp-contract=off (no FMA).
 *
 * Reference files restated (paths within the reference project):
 *   geometry parse   src/geometry/GeometryReader.cc:382-444, 515-607, 800-946
 *   site data        src/geometry/SiteDataBare.cc:24-172
 *   site order       src/geometry/LatticeData.cc:69-285, LatticeData.h:375-436,
 *                    src/geometry/VolumeTraverser.cc:59-84
 *   neighbour table  src/geometry/LatticeData.cc:366-443
 *   moments (SSE3)   src/lb/lattices/Lattice.h:51-110
 *   equilibrium      src/lb/lattices/Lattice.h:374-448, 933-948
 *   LBGK / TRT       src/lb/kernels/LBGK.h:32-72, src/lb/kernels/TRT.h:35-109
 *   LES + sponge     src/lb/kernels/LBGKLESSpongeLayer.h:27-182
 *   streamers        src/lb/streamers/StreamerTypeFactory.h:47-300,
 *                    SimpleCollideAndStream.h:38-68, SimpleBounceBackDelegate.h:27-44,
 *                    BouzidiFirdaousLallemandDelegate.h:44-93,
 *                    GuoZhengShiDelegate.h:127-321,
 *                    NashZerothOrderPressureDelegate.h:36-116, LaddIoletDelegate.h:37-126
 *   step phases      src/lb/lb.hpp:205-346
 *   iolets           src/lb/iolets/InOutLetCosine.cc:37-54,
 *                    InOutLetParabolicVelocity.cc:30-58, InOutLetWK3.cc:33-105,
 *                    InOutLetFileVelocity.cc:104-128,
 *                    InOutLetWomersleyVelocity.cc:15-41, src/util/Bessel.cc:17-43,
 *                    BoundaryValues.cc:20-224, BoundaryComms.cc:48-80
 *   macroscopic      src/lb/streamers/BaseStreamer.h:87-225,
 *                    src/lb/lattices/Lattice.h:1122-1156, 1353-1383
 */
#include "hb_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define Q ORC_Q

/* D3Q19 (src/lb/lattices/D3Q19.cc:15-33). */
static const int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int INV[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
static double CXD[Q], CYD[Q], CZD[Q], W[Q];
static const int* CV[3] = {CX, CY, CZ};
static const double CS2 = 1.0 / 3.0;
static const double PI_ = 3.14159265358979323846264338327950288;
static const double NO_VALUE = DBL_MAX;

static void init_tables(void) {
  for (int i = 0; i < Q; i++) {
    CXD[i] = (double)CX[i];
    CYD[i] = (double)CY[i];
    CZD[i] = (double)CZ[i];
    W[i] = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
  }
}

/* ------------------------------------------------------------------------- */
/* Lattice maths in the reference's SSE3 order.                               */
/* ------------------------------------------------------------------------- */

/* Lattice::CalculateDensityAndMomentum (SSE3): two lanes, f18 seeds the high lane,
 * even directions in the low lane, odd in the high lane, then a horizontal add. */
static inline void moments(const double* f, double* rho, double* mx, double* my, double* mz) {
  double dl = 0.0, dh = f[18];
  double xl = 0.0, xh = CXD[18] * f[18];
  double yl = 0.0, yh = CYD[18] * f[18];
  double zl = 0.0, zh = CZD[18] * f[18];
  for (int d = 0; d < 18; d += 2) {
    dl = dl + f[d];
    dh = dh + f[d + 1];
    xl = xl + CXD[d] * f[d];
    xh = xh + CXD[d + 1] * f[d + 1];
    yl = yl + CYD[d] * f[d];
    yh = yh + CYD[d + 1] * f[d + 1];
    zl = zl + CZD[d] * f[d];
    zh = zh + CZD[d + 1] * f[d + 1];
  }
  *rho = dl + dh;
  *mx = xl + xh;
  *my = yl + yh;
  *mz = zl + zh;
}

/* Lattice::CalculateFeq (SSE3 form; the odd last direction uses the same association). */
static inline void feq_calc(double rho, double mx, double my, double mz, double* feq) {
  const double th = (3. / 2.) * (mx * mx + my * my + mz * mz);
  const double d1 = 1. / rho;
  const double nh = (9. / 2.) * d1;
  for (int i = 0; i < Q; i++) {
    const double mde = CXD[i] * mx + CYD[i] * my + CZD[i] * mz;
    const double t1 = rho - th * d1;
    const double t2 = nh * (mde * mde);
    const double t3 = 3. * mde;
    feq[i] = W[i] * ((t1 + t2) + t3);
  }
}

typedef struct {
  double rho, mx, my, mz, ux, uy, uz, tau;
  double f[Q], feq[Q], fneq[Q], fpost[Q];
} hydro_t;

/* ------------------------------------------------------------------------- */
/* Geometry parse + lattice construction                                      */
/* ------------------------------------------------------------------------- */

struct orc_lattice {
  int64_t blocks[3], bs, dims[3];
  int64_t n;
  int64_t type_count[6];
  int32_t* grid;       /* dense [dims] -> contiguous index or -1 */
  int64_t* coords;     /* [n*3] */
  int64_t* nbr;        /* [n*19] */
  uint32_t* wall;      /* [n] */
  uint32_t* iolet;     /* [n] */
  int32_t* stype;      /* [n] 0 fluid, 1 inlet, 2 outlet (SiteType) */
  int32_t* iolet_id;   /* [n] */
  double* q;           /* [n*18] */
  double* normal;      /* [n*3] */
};

typedef struct {
  const unsigned char* p;
  size_t len, pos;
  int bad;
} xdr_t;

static uint32_t xdr_u32(xdr_t* x) {
  if (x->pos + 4 > x->len) {
    x->bad = 1;
    return 0;
  }
  const unsigned char* b = x->p + x->pos;
  x->pos += 4;
  return ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | (uint32_t)b[3];
}

static float xdr_f32(xdr_t* x) {
  uint32_t u = xdr_u32(x);
  float f;
  memcpy(&f, &u, 4);
  return f;
}

/* Per fluid site as read (GeometrySite): only the 18 D3Q19 links are kept. */
typedef struct {
  uint8_t type[18];
  int32_t iolet_id[18];
  float dist[18];
  int normal_avail;
  float normal[3];
} read_site_t;

/* .gmy displacement order (src/io/formats/geometry.cc:16-52). */
static int gmy_disp[26][3];
static int gmy_to_q[26];

static void init_gmy_tables(void) {
  int k = 0;
  for (int dx = -1; dx <= 1; dx++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dz = -1; dz <= 1; dz++) {
        if (!dx && !dy && !dz) continue;
        gmy_disp[k][0] = dx;
        gmy_disp[k][1] = dy;
        gmy_disp[k][2] = dz;
        gmy_to_q[k] = -1;
        for (int d = 1; d < Q; d++)
          if (CX[d] == dx && CY[d] == dy && CZ[d] == dz) gmy_to_q[k] = d;
        k++;
      }
}

static void seterr(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", msg);
}

void orc_lattice_free(orc_lattice* l) {
  if (!l) return;
  free(l->grid);
  free(l->coords);
  free(l->nbr);
  free(l->wall);
  free(l->iolet);
  free(l->stype);
  free(l->iolet_id);
  free(l->q);
  free(l->normal);
  free(l);
}

int orc_lattice_load(const char* path, orc_lattice** out, char* err, int errlen) {
  init_tables();
  init_gmy_tables();
  *out = NULL;
  FILE* fh = fopen(path, "rb");
  if (!fh) {
    seterr(err, errlen, "cannot open geometry file");
    return -1;
  }
  fseek(fh, 0, SEEK_END);
  long flen = ftell(fh);
  fseek(fh, 0, SEEK_SET);
  unsigned char* buf = (unsigned char*)malloc((size_t)flen);
  if (fread(buf, 1, (size_t)flen, fh) != (size_t)flen) {
    fclose(fh);
    free(buf);
    seterr(err, errlen, "short read");
    return -1;
  }
  fclose(fh);

  xdr_t x = {buf, (size_t)flen, 0, 0};
  uint32_t hlb = xdr_u32(&x), gmy = xdr_u32(&x), ver = xdr_u32(&x);
  if (hlb != 0x686c6221u || gmy != 0x676d7904u || ver != 4u) {
    free(buf);
    seterr(err, errlen, "bad preamble (magic numbers or version)");
    return -2;
  }
  orc_lattice* l = (orc_lattice*)calloc(1, sizeof(orc_lattice));
  for (int d = 0; d < 3; d++) l->blocks[d] = xdr_u32(&x);
  l->bs = xdr_u32(&x);
  (void)xdr_u32(&x); /* padding */
  const int64_t bs = l->bs, bs3 = bs * bs * bs;
  const int64_t nblocks = l->blocks[0] * l->blocks[1] * l->blocks[2];
  for (int d = 0; d < 3; d++) l->dims[d] = l->blocks[d] * bs;
  uint32_t* hdr = (uint32_t*)malloc(sizeof(uint32_t) * 3 * (size_t)nblocks);
  x.pos = 32;
  for (int64_t b = 0; b < nblocks; b++) {
    hdr[3 * b] = xdr_u32(&x);
    hdr[3 * b + 1] = xdr_u32(&x);
    hdr[3 * b + 2] = xdr_u32(&x);
  }
  if (x.bad) {
    free(buf);
    free(hdr);
    orc_lattice_free(l);
    seterr(err, errlen, "truncated header");
    return -3;
  }
  /* Parse every non-empty block into read sites. */
  int64_t total_fluid = 0;
  for (int64_t b = 0; b < nblocks; b++) total_fluid += hdr[3 * b];
  read_site_t* rs = (read_site_t*)calloc((size_t)(total_fluid > 0 ? total_fluid : 1), sizeof(read_site_t));
  int64_t* block_first = (int64_t*)malloc(sizeof(int64_t) * (size_t)nblocks);
  int32_t* local_fluid = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nblocks * bs3 > 0 ? nblocks * bs3 : 1));
  size_t off = (size_t)(32 + 12 * nblocks);
  int64_t nf = 0;
  unsigned char* raw = NULL;
  size_t rawcap = 0;
  int rc = 0;
  for (int64_t b = 0; b < nblocks && !rc; b++) {
    block_first[b] = nf;
    for (int64_t s = 0; s < bs3; s++) local_fluid[b * bs3 + s] = -1;
    if (hdr[3 * b] == 0) continue;
    uint32_t cb = hdr[3 * b + 1], ub = hdr[3 * b + 2];
    if (off + cb > (size_t)flen) {
      rc = -4;
      seterr(err, errlen, "truncated block data");
      break;
    }
    if (ub > rawcap) {
      rawcap = ub;
      raw = (unsigned char*)realloc(raw, rawcap);
    }
    uLongf dl = ub;
    if (uncompress(raw, &dl, buf + off, cb) != Z_OK) {
      rc = -5;
      seterr(err, errlen, "decompression error for block");
      break;
    }
    off += cb;
    xdr_t bx = {raw, (size_t)dl, 0, 0};
    int64_t nfb = 0;
    for (int64_t s = 0; s < bs3; s++) {
      uint32_t isf = xdr_u32(&bx);
      if (!isf) continue;
      read_site_t* r = &rs[nf];
      for (int d = 0; d < 18; d++) {
        r->type[d] = 0;
        r->iolet_id[d] = -1;
        r->dist[d] = -1.0f;
      }
      int gmy_wall = 0;
      for (int k = 0; k < 26; k++) {
        uint32_t t = xdr_u32(&bx);
        float dist = -1.0f;
        int32_t iid = -1;
        if (t == 1) {
          gmy_wall = 1;
          dist = xdr_f32(&bx);
        } else if (t != 0) {
          iid = (int32_t)xdr_u32(&bx);
          dist = xdr_f32(&bx);
        }
        int d = gmy_to_q[k];
        if (d > 0) {
          r->type[d - 1] = (uint8_t)t;
          r->iolet_id[d - 1] = iid;
          r->dist[d - 1] = dist;
        }
      }
      uint32_t na = xdr_u32(&bx);
      r->normal_avail = (na == 1u);
      if (r->normal_avail != gmy_wall) {
        rc = -6;
        seterr(err, errlen, "Malformed GMY file: wall normal availability does not match wall links");
        break;
      }
      if (r->normal_avail) {
        r->normal[0] = xdr_f32(&bx);
        r->normal[1] = xdr_f32(&bx);
        r->normal[2] = xdr_f32(&bx);
      }
      local_fluid[b * bs3 + s] = (int32_t)nf;
      nf++;
      nfb++;
    }
    if (bx.bad && !rc) {
      rc = -7;
      seterr(err, errlen, "truncated site record");
    }
    if (!rc && nfb != (int64_t)hdr[3 * b]) {
      rc = -8;
      seterr(err, errlen, "block fluid-site count does not match its header");
    }
  }
  free(raw);
  free(buf);
  if (rc) {
    free(rs);
    free(block_first);
    free(local_fluid);
    free(hdr);
    orc_lattice_free(l);
    return rc;
  }

  /* Classify (SiteData ctor) and bin by collision type in block traversal order. */
  int64_t n = nf;
  l->n = n;
  int32_t* rs_type = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int64_t* order_rs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t* order_pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)(3 * (n > 0 ? n : 1)));
  uint32_t* rs_wall = (uint32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(uint32_t));
  uint32_t* rs_iolet = (uint32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(uint32_t));
  int32_t* rs_stype = (int32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
  int32_t* rs_iid = (int32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
  for (int64_t i = 0; i < n; i++) {
    const read_site_t* r = &rs[i];
    uint32_t w = 0, io = 0;
    int had_in = 0, had_out = 0;
    int32_t iid = -1;
    for (int d = 1; d <= 18; d++) {
      int t = r->type[d - 1];
      if (t == 1) w |= 1u << (d - 1);
      else if (t == 2 || t == 3) io |= 1u << (d - 1);
      if (t == 2) {
        iid = r->iolet_id[d - 1];
        had_in = 1;
      } else if (t == 3) {
        iid = r->iolet_id[d - 1];
        had_out = 1;
      }
    }
    int st = had_in ? 1 : (had_out ? 2 : 0);
    rs_wall[i] = w;
    rs_iolet[i] = io;
    rs_stype[i] = st;
    rs_iid[i] = iid;
    /* collision type: FLUID 0, WALL 1, INLET 2, OUTLET 3, INLET|WALL 4, OUTLET|WALL 5 */
    rs_type[i] = w == 0 ? (st == 0 ? 0 : (st == 1 ? 2 : 3)) : (st == 0 ? 1 : (st == 1 ? 4 : 5));
  }
  for (int t = 0; t < 6; t++) l->type_count[t] = 0;
  for (int64_t i = 0; i < n; i++) l->type_count[rs_type[i]]++;
  int64_t start[6];
  start[0] = 0;
  for (int t = 1; t < 6; t++) start[t] = start[t - 1] + l->type_count[t - 1];
  int64_t fill[6];
  for (int t = 0; t < 6; t++) fill[t] = start[t];
  l->grid = (int32_t*)malloc(sizeof(int32_t) * (size_t)(l->dims[0] * l->dims[1] * l->dims[2]));
  for (int64_t g = 0; g < l->dims[0] * l->dims[1] * l->dims[2]; g++) l->grid[g] = -1;
  /* Block traversal: x-major over blocks, z fastest; same inside a block. */
  for (int64_t bxi = 0; bxi < l->blocks[0]; bxi++)
    for (int64_t byi = 0; byi < l->blocks[1]; byi++)
      for (int64_t bzi = 0; bzi < l->blocks[2]; bzi++) {
        int64_t b = (bxi * l->blocks[1] + byi) * l->blocks[2] + bzi;
        if (hdr[3 * b] == 0) continue;
        for (int64_t sx = 0; sx < bs; sx++)
          for (int64_t sy = 0; sy < bs; sy++)
            for (int64_t sz = 0; sz < bs; sz++) {
              int64_t s = (sx * bs + sy) * bs + sz;
              int32_t ri = local_fluid[b * bs3 + s];
              if (ri < 0) continue;
              int64_t c = fill[rs_type[ri]]++;
              order_rs[c] = ri;
              order_pos[3 * c] = bxi * bs + sx;
              order_pos[3 * c + 1] = byi * bs + sy;
              order_pos[3 * c + 2] = bzi * bs + sz;
            }
      }
  free(hdr);
  free(block_first);
  free(local_fluid);
  l->coords = (int64_t*)malloc(sizeof(int64_t) * (size_t)(3 * (n > 0 ? n : 1)));
  l->wall = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
  l->iolet = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
  l->stype = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  l->iolet_id = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  l->q = (double*)malloc(sizeof(double) * (size_t)(18 * (n > 0 ? n : 1)));
  l->normal = (double*)malloc(sizeof(double) * (size_t)(3 * (n > 0 ? n : 1)));
  for (int64_t c = 0; c < n; c++) {
    int64_t ri = order_rs[c];
    const read_site_t* r = &rs[ri];
    for (int d = 0; d < 3; d++) l->coords[3 * c + d] = order_pos[3 * c + d];
    l->grid[(order_pos[3 * c] * l->dims[1] + order_pos[3 * c + 1]) * l->dims[2] + order_pos[3 * c + 2]] = (int32_t)c;
    l->wall[c] = rs_wall[ri];
    l->iolet[c] = rs_iolet[ri];
    l->stype[c] = rs_stype[ri];
    l->iolet_id[c] = rs_iid[ri];
    for (int d = 0; d < 18; d++) l->q[18 * c + d] = (double)r->dist[d];
    if (r->normal_avail) {
      /* Vector3D<float>::GetNormalised in float arithmetic (LatticeData.cc:252-254). */
      float nx = r->normal[0], ny = r->normal[1], nz = r->normal[2];
      if (nx == 0.0f && ny == 0.0f && nz == 0.0f) {
        l->normal[3 * c] = 0.0;
        l->normal[3 * c + 1] = 0.0;
        l->normal[3 * c + 2] = 0.0;
      } else {
        float m2 = nx * nx + ny * ny + nz * nz;
        float m = sqrtf(m2);
        l->normal[3 * c] = (double)(nx / m);
        l->normal[3 * c + 1] = (double)(ny / m);
        l->normal[3 * c + 2] = (double)(nz / m);
      }
    } else {
      float nv = (float)HUGE_VAL; /* NO_VALUE narrowed to float */
      l->normal[3 * c] = l->normal[3 * c + 1] = l->normal[3 * c + 2] = (double)nv;
    }
  }
  free(rs);
  free(order_rs);
  free(order_pos);
  free(rs_type);
  free(rs_wall);
  free(rs_iolet);
  free(rs_stype);
  free(rs_iid);

  /* Neighbour table: contig(x+c_d)*19+d, or the rubbish slot N*19. */
  l->nbr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(Q * (n > 0 ? n : 1)));
  for (int64_t c = 0; c < n; c++) {
    l->nbr[Q * c] = Q * c;
    for (int d = 1; d < Q; d++) {
      int64_t px = l->coords[3 * c] + CX[d], py = l->coords[3 * c + 1] + CY[d], pz = l->coords[3 * c + 2] + CZ[d];
      int64_t t = n * Q;
      if (px >= 0 && py >= 0 && pz >= 0 && px < l->dims[0] && py < l->dims[1] && pz < l->dims[2]) {
        int32_t g = l->grid[(px * l->dims[1] + py) * l->dims[2] + pz];
        if (g >= 0) t = (int64_t)g * Q + d;
      }
      l->nbr[Q * c + d] = t;
    }
  }
  *out = l;
  return 0;
}

int64_t orc_site_count(const orc_lattice* l) { return l->n; }
void orc_type_counts(const orc_lattice* l, int64_t counts[6]) {
  for (int t = 0; t < 6; t++) counts[t] = l->type_count[t];
}
void orc_dims(const orc_lattice* l, int64_t blocks[3], int64_t* block_size) {
  for (int d = 0; d < 3; d++) blocks[d] = l->blocks[d];
  *block_size = l->bs;
}
void orc_get_coords(const orc_lattice* l, int64_t* xyz) { memcpy(xyz, l->coords, sizeof(int64_t) * 3 * (size_t)l->n); }
void orc_get_neighbours(const orc_lattice* l, int64_t* nbr) { memcpy(nbr, l->nbr, sizeof(int64_t) * Q * (size_t)l->n); }
void orc_get_sitedata(const orc_lattice* l, uint32_t* wall, uint32_t* iolet, int32_t* type, int32_t* iid) {
  memcpy(wall, l->wall, sizeof(uint32_t) * (size_t)l->n);
  memcpy(iolet, l->iolet, sizeof(uint32_t) * (size_t)l->n);
  memcpy(type, l->stype, sizeof(int32_t) * (size_t)l->n);
  memcpy(iid, l->iolet_id, sizeof(int32_t) * (size_t)l->n);
}
void orc_get_wall_distance(const orc_lattice* l, double* q) { memcpy(q, l->q, sizeof(double) * 18 * (size_t)l->n); }
void orc_get_wall_normal(const orc_lattice* l, double* nrm) { memcpy(nrm, l->normal, sizeof(double) * 3 * (size_t)l->n); }

/* ------------------------------------------------------------------------- */
/* Iolets                                                                     */
/* ------------------------------------------------------------------------- */

typedef struct {
  orc_iolet cfg;
  float normal_f[3];        /* the normal narrowed to float (Nash delegate) */
  int dir0;                 /* direction closest to the normal */
  int64_t centre;           /* centre site (first site within +-1 of the position) */
  double min_density;       /* minimumSimulationDensity */
  /* WK3 state */
  double density, density_new, flow, flow_old, flow_new;
  int64_t count;
} iolet_t;

struct orc_sim {
  const orc_lattice* lat;
  orc_params p;
  double omega;
  double* f_old;
  double* f_new;
  double* rho;
  double* u;
  double* wss;
  double* stress;           /* [n*17] stress caches of the last macro step (allocated at the first) */
  double* vtau;
  int nthreads;
  uint64_t t;               /* 1-based time step */
  iolet_t io[2][16];
  int nio[2];
  /* per site, for the ordered iolet coupling pass */
  double* cpl_u;            /* [n*3] */
  int8_t* cpl_flag;         /* [n] 1 if the site couples this step */
  int status;
};

static double cosine_density(const iolet_t* io, uint64_t t0) {
  /* InOutLetCosine::GetDensity with the 0-indexed step (BoundaryValues.cc:211-214). */
  const double w = 2.0 * PI_ / io->cfg.period;
  const double target = io->cfg.density_mean + io->cfg.density_amp * cos(w * (double)t0 + io->cfg.phase);
  if (t0 >= io->cfg.warmup) return target;
  const double fac = ((double)t0) / ((double)io->cfg.warmup);
  return fac * target + (1. - fac) * io->min_density;
}

static double iolet_density(const iolet_t* io, uint64_t t0) {
  if (io->cfg.kind == ORC_IOLET_COSINE) return cosine_density(io, t0);
  if (io->cfg.kind == ORC_IOLET_WK3 || io->cfg.kind == ORC_IOLET_WK2) return io->density;
  if (io->cfg.kind == ORC_IOLET_FILE) /* InOutLetFile::GetDensity: densityTable[timeStep] */
    return io->cfg.table[t0 < io->cfg.table_len ? t0 : io->cfg.table_len - 1];
  return 1.0; /* InOutLetVelocity::GetDensity */
}

static int is_windkessel(const iolet_t* io) { return io->cfg.kind == ORC_IOLET_WK3 || io->cfg.kind == ORC_IOLET_WK2; }

/* InOutLetParabolicVelocity::GetVelocity.  Returns 0, or -1 for a point
 * outside the iolet radius (the reference exits with code 16). */
static int parabolic_velocity(const iolet_t* io, const double x[3], uint64_t t1, double v[3]) {
  const double dx = x[0] - io->cfg.position[0], dy = x[1] - io->cfg.position[1], dz = x[2] - io->cfg.position[2];
  const double* n = io->cfg.normal;
  const double z = dx * n[0] + dy * n[1] + dz * n[2];
  const double rsq = (dx * dx + dy * dy + dz * dz) - z * z;
  const double r2a2 = rsq / (io->cfg.radius * io->cfg.radius);
  if (r2a2 > 1.0) return -1;
  double mx = io->cfg.max_speed;
  if (t1 < io->cfg.warmup) mx *= (double)t1 / (double)io->cfg.warmup;
  const double s = mx * (1. - r2a2);
  v[0] = n[0] * s;
  v[1] = n[1] * s;
  v[2] = n[2] * s;
  return 0;
}

/* InOutLetFileVelocity::GetVelocity: the parabolic profile with the peak speed
 * velocityTable[t] (steps past the table take its last entry). */
static int file_velocity(const iolet_t* io, const double x[3], uint64_t t1, double v[3]) {
  const double dx = x[0] - io->cfg.position[0], dy = x[1] - io->cfg.position[1], dz = x[2] - io->cfg.position[2];
  const double* n = io->cfg.normal;
  const double z = dx * n[0] + dy * n[1] + dz * n[2];
  const double rsq = (dx * dx + dy * dy + dz * dz) - z * z;
  const double r2a2 = rsq / (io->cfg.radius * io->cfg.radius);
  if (r2a2 > 1.0) return -1;
  const double mx = io->cfg.table[t1 < io->cfg.table_len ? t1 : io->cfg.table_len - 1];
  const double s = mx * (1. - r2a2);
  v[0] = n[0] * s;
  v[1] = n[1] * s;
  v[2] = n[2] * s;
  return 0;
}

/* util::BesselJ0ComplexArgument: the power series of J0, summed until the squared
 * modulus of the last term is at most tol_sq, in the reference's operation order. */
static double complex bessel_j0(double complex z, double tol_sq) {
  double complex sum = 1.0, zpow = 1.0, term = 1.0;
  double fact = 1;
  for (unsigned k = 1; creal(term) * creal(term) + cimag(term) * cimag(term) > tol_sq; ++k) {
    fact *= k;
    zpow *= -0.25 * z * z;
    term = zpow / (fact * fact);
    sum += term;
  }
  return sum;
}

void orc_bessel_j0(double re, double im, double out[2]) {
  const double complex j = bessel_j0(CMPLX(re, im), 1e-12);
  out[0] = creal(j);
  out[1] = cimag(j);
}

/* InOutLetWomersleyVelocity::GetVelocity:
 *   v = -normal Re[ G / (rho omega) (1 - J0(i^(3/2) alpha r / R) / J0(i^(3/2) alpha)) exp(i omega t) ]
 * with rho = 1.  i^(3/2) is std::pow(complex i, 1.5) of the C++ library the
 * reference builds with: polar(exp(1.5 Re log i), 1.5 Im log i). */
static void womersley_velocity(const iolet_t* io, const double x[3], uint64_t t1, double v[3]) {
  const double dx = x[0] - io->cfg.position[0], dy = x[1] - io->cfg.position[1], dz = x[2] - io->cfg.position[2];
  const double* n = io->cfg.normal;
  const double z = dx * n[0] + dy * n[1] + dz * n[2];
  const double r = sqrt((dx * dx + dy * dy + dz * dz) - z * z);
  const double omega = 2.0 * PI_ / io->cfg.period;
  const double density = 1.0;
  const double complex lg = clog(CMPLX(0.0, 1.0));
  const double rho = exp(1.5 * creal(lg)), th = 1.5 * cimag(lg);
  const double complex i32 = CMPLX(rho * cos(th), rho * sin(th));
  const double complex numer = bessel_j0(i32 * io->cfg.womersley_number * r / io->cfg.radius, 1e-12);
  const double complex denom = bessel_j0(i32 * io->cfg.womersley_number, 1e-12);
  const double complex amp = io->cfg.pressure_gradient_amplitude / (density * omega) * (1.0 - numer / denom);
  const double speed = creal(amp * cexp(CMPLX(0.0, omega * (double)t1)));
  v[0] = n[0] * -speed;
  v[1] = n[1] * -speed;
  v[2] = n[2] * -speed;
}

static int is_velocity_iolet(const iolet_t* io) {
  return io->cfg.kind == ORC_IOLET_PARABOLIC || io->cfg.kind == ORC_IOLET_FILE_VELOCITY || io->cfg.kind == ORC_IOLET_WOMERSLEY;
}

/* The velocity iolets' GetVelocity; 0, or -1 outside a parabolic profile's radius. */
static int iolet_velocity(const iolet_t* io, const double x[3], uint64_t t1, double v[3]) {
  if (io->cfg.kind == ORC_IOLET_WOMERSLEY) {
    womersley_velocity(io, x, t1, v);
    return 0;
  }
  if (io->cfg.kind == ORC_IOLET_FILE_VELOCITY) return file_velocity(io, x, t1, v);
  return parabolic_velocity(io, x, t1, v);
}

int orc_iolet_velocity(const orc_iolet* cfg, const double x[3], uint64_t t, double v[3]) {
  iolet_t io;
  memset(&io, 0, sizeof(io));
  io.cfg = *cfg;
  if (!is_velocity_iolet(&io)) return -2;
  return iolet_velocity(&io, x, t, v);
}

static void sort_dirs_close_to_normal(iolet_t* io) {
  /* Nash/Ladd SortDirectionsCloseToIOletNormal: the direction minimising
   * |c_k/|c_k| - n|^2 (the zero vector stays zero when normalised). */
  double best = DBL_MAX;
  int bi = 0;
  for (int k = 0; k < Q; k++) {
    double cx = CXD[k], cy = CYD[k], cz = CZD[k];
    double m2 = cx * cx + cy * cy + cz * cz;
    if (m2 != 0.0) {
      double m = sqrt(m2);
      cx /= m;
      cy /= m;
      cz /= m;
    }
    double ex = cx - io->cfg.normal[0], ey = cy - io->cfg.normal[1], ez = cz - io->cfg.normal[2];
    double dist = ex * ex + ey * ey + ez * ez;
    if (dist < best) {
      best = dist;
      bi = k;
    }
  }
  io->dir0 = bi;
}

/* ------------------------------------------------------------------------- */
/* Simulation                                                                 */
/* ------------------------------------------------------------------------- */

void orc_sim_free(orc_sim* s) {
  if (!s) return;
  free(s->f_old);
  free(s->f_new);
  free(s->rho);
  free(s->u);
  free(s->wss);
  free(s->stress);
  free(s->vtau);
  free(s->cpl_u);
  free(s->cpl_flag);
  free(s);
}

void orc_sim_set_threads(orc_sim* s, int nthreads) { s->nthreads = nthreads > 0 ? nthreads : 1; }

int orc_sim_create(const orc_lattice* lat, const orc_params* p, orc_sim** out, char* err, int errlen) {
  init_tables();
  *out = NULL;
  if ((p->kernel == ORC_LBGKLES || p->kernel == ORC_LBGKSL || p->kernel == ORC_TRTSL) && p->wall == ORC_GZS) {
    /* The GZS virtual-node collision reads a relaxation time that the sponge-layer
     * kernels (LES or not) never set on the wall node's HydroVars. */
    seterr(err, errlen, "GZS walls with a sponge-layer kernel are not supported");
    return -1;
  }
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  s->lat = lat;
  s->p = *p;
  s->omega = -1.0 / p->tau;
  s->nthreads = 1;
  s->t = p->initial_step ? p->initial_step : 1;
  const int64_t n = lat->n;
  s->f_old = (double*)malloc(sizeof(double) * (size_t)(n * Q + 1));
  s->f_new = (double*)malloc(sizeof(double) * (size_t)(n * Q + 1));
  s->rho = (double*)calloc((size_t)(n + 1), sizeof(double));
  s->u = (double*)calloc((size_t)(3 * n + 1), sizeof(double));
  s->wss = (double*)calloc((size_t)(n + 1), sizeof(double));
  s->cpl_u = (double*)calloc((size_t)(3 * n + 1), sizeof(double));
  s->cpl_flag = (int8_t*)calloc((size_t)(n + 1), 1);
  /* Equilibrium initial condition (InitialCondition.hpp:29-49). */
  double feq[Q];
  feq_calc(p->initial_density, 0.0, 0.0, 0.0, feq);
  for (int64_t i = 0; i < n; i++)
    for (int d = 0; d < Q; d++) s->f_old[i * Q + d] = s->f_new[i * Q + d] = feq[d];
  s->f_old[n * Q] = s->f_new[n * Q] = 0.0;

  /* Iolets: copy, minimum density over all (LBM::PrepareBoundaryObjects), sort, centre. */
  s->nio[0] = p->n_inlets;
  s->nio[1] = p->n_outlets;
  double mind = DBL_MAX;
  for (int g = 0; g < 2; g++)
    for (int k = 0; k < s->nio[g]; k++) {
      iolet_t* io = &s->io[g][k];
      io->cfg = g == 0 ? p->inlets[k] : p->outlets[k];
      /* GetDensityMin: cosine mean - amplitude, file its table's minimum, others 1 */
      double dmin = io->cfg.kind == ORC_IOLET_COSINE ? io->cfg.density_mean - io->cfg.density_amp
                    : io->cfg.kind == ORC_IOLET_FILE ? io->cfg.density_min : 1.0;
      if (dmin < mind) mind = dmin;
      for (int d = 0; d < 3; d++) io->normal_f[d] = (float)io->cfg.normal[d];
      sort_dirs_close_to_normal(io);
      io->centre = -1;
      for (int64_t i = 0; i < n; i++) {
        int in = 1;
        for (int d = 0; d < 3; d++) {
          double c = (double)lat->coords[3 * i + d];
          if (!(c >= io->cfg.position[d] - 1.0 && c <= io->cfg.position[d] + 1.0)) in = 0;
        }
        if (in) {
          io->centre = i;
          break;
        }
      }
      io->density = 1.0;
      io->density_new = 1.0;
      io->flow = io->flow_old = io->flow_new = 0.0;
      io->count = 0;
    }
  for (int g = 0; g < 2; g++)
    for (int k = 0; k < s->nio[g]; k++) s->io[g][k].min_density = mind;

  /* Sponge relaxation time per site (LBGKLESSpongeLayer::InitState; the same in
   * LBGKSpongeLayer.h:88-116 and TRTSpongeLayer.h:124-151).  `siteLocation -
   * outletPositions[j]` is Vector3D<site_t>::operator-, whose argument is the
   * position converted to integers by truncation (src/util/Vector3D.h:238-243,
   * 396): the squared distance is an integer sum. */
  if (p->kernel == ORC_LBGKLES || p->kernel == ORC_LBGKSL || p->kernel == ORC_TRTSL) {
    s->vtau = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    const double width = p->sponge_width, widthsq = width * width;
    for (int64_t i = 0; i < n; i++) {
      double vr = 1.0;
      for (int k = 0; k < p->n_outlets; k++) {
        const int64_t dx = (int64_t)lat->coords[3 * i] - (int64_t)p->outlets[k].position[0];
        const int64_t dy = (int64_t)lat->coords[3 * i + 1] - (int64_t)p->outlets[k].position[1];
        const int64_t dz = (int64_t)lat->coords[3 * i + 2] - (int64_t)p->outlets[k].position[2];
        const double distsq = (double)(dx * dx + dy * dy + dz * dz);
        const double dist = sqrt(distsq);
        if (distsq <= widthsq)
          vr *= 1.0 + (p->viscosity_ratio - 1.0) * (dist / width - 1.0) * (dist / width - 1.0);
      }
      s->vtau[i] = vr * (p->tau - 0.5) + 0.5;
    }
  }
  *out = s;
  return 0;
}

uint64_t orc_sim_time_step(const orc_sim* s) { return s->t; }

void orc_sim_get_f(const orc_sim* s, double* f) { memcpy(f, s->f_old, sizeof(double) * Q * (size_t)s->lat->n); }

void orc_sim_set_f(orc_sim* s, const double* f) {
  memcpy(s->f_old, f, sizeof(double) * Q * (size_t)s->lat->n);
  memcpy(s->f_new, f, sizeof(double) * Q * (size_t)s->lat->n);
}

void orc_sim_get_macro(const orc_sim* s, double* rho, double* u, double* wss) {
  const int64_t n = s->lat->n;
  if (rho) memcpy(rho, s->rho, sizeof(double) * (size_t)n);
  if (u) memcpy(u, s->u, sizeof(double) * 3 * (size_t)n);
  if (wss) memcpy(wss, s->wss, sizeof(double) * (size_t)n);
}

int orc_sim_get_stress(const orc_sim* s, int field, double* out) {
  static const int first[6] = {0, 1, 2, 8, 11, 14}, len[6] = {1, 1, 6, 3, 3, 3};
  if (field < 0 || field > 5 || !s->stress) return -1;
  const int64_t n = s->lat->n;
  for (int64_t i = 0; i < n; i++)
    for (int k = 0; k < len[field]; k++) out[i * len[field] + k] = s->stress[17 * i + first[field] + k];
  return 0;
}

void orc_sim_get_wk3(const orc_sim* s, int group, int index, double st[4]) {
  const iolet_t* io = &s->io[group][index];
  st[0] = io->density;
  st[1] = io->density_new;
  st[2] = io->flow;
  st[3] = io->flow_old;
}

void orc_sim_get_vtau(const orc_sim* s, double* vtau) {
  if (s->vtau) memcpy(vtau, s->vtau, sizeof(double) * (size_t)s->lat->n);
}

/* Kernel: density, momentum, equilibrium, non-equilibrium (+ LES tau). */
static inline void pre_collision(const orc_sim* s, int64_t i, hydro_t* h) {
  moments(h->f, &h->rho, &h->mx, &h->my, &h->mz);
  h->ux = h->mx / h->rho;
  h->uy = h->my / h->rho;
  h->uz = h->mz / h->rho;
  feq_calc(h->rho, h->mx, h->my, h->mz, h->feq);
  for (int d = 0; d < Q; d++) h->fneq[d] = h->f[d] - h->feq[d];
  h->tau = s->p.tau;
  if (s->p.kernel == ORC_LBGKLES) {
    /* compute_tau_smagorinsky (dx = dt = rho1 = 1, C_smag = 0.1) */
    const double tau0 = s->p.tau, C = 1.0, rho1 = 1.0, csmag = 0.1;
    double q12 = 0.0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double qij = 0.0;
        for (int v = 0; v < Q; v++) qij += (double)(CV[a][v] * CV[b][v]) * h->fneq[v];
        q12 += qij * qij;
      }
    q12 = sqrt(q12);
    const double tau_les =
        1. / 2. * (tau0 + sqrt((tau0 * rho1 * C) * (tau0 * rho1 * C) + 18.0 * 1.4142135623730950488016887242097 * rho1 * csmag * csmag * q12) / (rho1 * C));
    const uint64_t ts = s->t;
    const uint64_t life = s->p.sponge_lifetime;
    const double vt = s->vtau[i];
    if (ts <= life / 2) {
      h->tau = (vt == tau0) ? tau_les : vt;
    } else if (ts < life) {
      h->tau = (tau_les - vt) * 2.0 / (double)life * (double)ts + (2.0 * vt - tau_les);
    } else {
      h->tau = tau_les;
    }
  } else if (s->p.kernel == ORC_LBGKSL || s->p.kernel == ORC_TRTSL) {
    /* CalculateTau (LBGKSpongeLayer.h:124-140, TRTSpongeLayer.h:157-172): the sponge
     * time for the first half of its lifetime, then a linear return to tau0. */
    const double tau0 = s->p.tau;
    const uint64_t ts = s->t;
    const uint64_t life = s->p.sponge_lifetime;
    const double vt = s->vtau[i];
    if (ts <= life / 2) {
      h->tau = vt;
    } else if (ts < life) {
      h->tau = (tau0 - vt) * 2.0 / (double)life * (double)ts + (2.0 * vt - tau0);
    } else {
      h->tau = tau0;
    }
  }
}

/* Collision on (f, fneq) into fpost; uses the kernel's own relaxation times. */
static inline void collide(const orc_sim* s, const double* f, const double* fneq, double tau_site, double* fpost) {
  if (s->p.kernel == ORC_LBGK) {
    const double om = s->omega;
    for (int d = 0; d < Q; d++) fpost[d] = f[d] + fneq[d] * om;
  } else if (s->p.kernel == ORC_TRT) {
    const double lambda = s->p.relaxation_parameter;
    const double tp = s->p.tau;
    const double op = s->omega;
    const double tm = 0.5 + lambda / (tp - 0.5);
    const double om = -1.0 / tm;
    fpost[0] = f[0] + op * fneq[0];
    for (int i = 0; i < Q; i++) {
      const int ib = INV[i];
      if (ib < i) continue;
      const double sym = 0.5 * op * (fneq[i] + fneq[ib]);
      const double asym = 0.5 * om * (fneq[i] - fneq[ib]);
      fpost[i] = f[i] + sym + asym;
      fpost[ib] = f[ib] + sym - asym;
    }
  } else if (s->p.kernel == ORC_TRTSL) {
    /* TRTSpongeLayer::DoCollide (TRTSpongeLayer.h:86-115): the symmetric rate stays
     * the global omega, the antisymmetric one follows the site's sponge tau. */
    const double lambda = s->p.relaxation_parameter;
    const double op = s->omega;
    const double tm = 0.5 + lambda / (tau_site - 0.5);
    const double om = -1.0 / tm;
    fpost[0] = f[0] + op * fneq[0];
    for (int i = 0; i < Q; i++) {
      const int ib = INV[i];
      if (ib < i) continue;
      const double sym = 0.5 * op * (fneq[i] + fneq[ib]);
      const double asym = 0.5 * om * (fneq[i] - fneq[ib]);
      fpost[i] = f[i] + sym + asym;
      fpost[ib] = f[ib] + sym - asym;
    }
  } else {
    const double om = -1.0 / tau_site;
    for (int d = 0; d < Q; d++) fpost[d] = f[d] + fneq[d] * om;
  }
}

static inline int has_wall(const orc_lattice* l, int64_t i, int d) { return d > 0 && (l->wall[i] >> (d - 1)) & 1u; }
static inline int has_iolet(const orc_lattice* l, int64_t i, int d) { return d > 0 && (l->iolet[i] >> (d - 1)) & 1u; }

static inline int site_ctype(const orc_lattice* l, int64_t i) {
  const int w = l->wall[i] != 0, st = l->stype[i];
  return !w ? (st == 0 ? 0 : (st == 1 ? 2 : 3)) : (st == 0 ? 1 : (st == 1 ? 4 : 5));
}

/* Wall-shear-stress magnitude (Lattice::CalculateWallShearStressMagnitude). */
static double wss_mag(double tau, const double* fpost, const double* f, const double* nor) {
  double pi[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b <= a; b++) {
      pi[a][b] = 0.0;
      for (int l = 0; l < Q; l++) pi[a][b] += (fpost[l] - f[l]) * (double)CV[a][l] * (double)CV[b][l];
      pi[a][b] *= -(tau - 0.5);
    }
  for (int a = 0; a < 3; a++)
    for (int b = a + 1; b < 3; b++) pi[a][b] = pi[b][a];
  double sv[3] = {0.0, 0.0, 0.0}, sq = 0.0, ns = 0.0;
  for (int a = 0; a < 3; a++) {
    for (int b = 0; b < 3; b++) sv[a] += pi[a][b] * nor[b];
    sq += sv[a] * sv[a];
    ns += sv[a] * nor[a];
  }
  return sqrt(sq - ns * ns);
}

/* Stress caches of one site (BaseStreamer::UpdateMinsAndMaxes,
 * src/lb/streamers/BaseStreamer.h:123-217), each from CalculatePiTensor
 * (src/lb/lattices/Lattice.h:1353-1383) in the reference's order:
 * o[0] CalculateVonMisesStress (:983-1002), o[1] CalculateShearRate (:1159-1175),
 * o[2..7] CalculateStressTensor (:1096-1112) as xx, xy, xz, yy, yz, zz,
 * o[8..10] CalculateTractionOnAPoint (:1017-1028; Matrix3D::timesVector,
 * src/util/Matrix3D.cc:45-55), o[11..13] CalculateTangentialProjectionTraction
 * (:1045-1057), o[14..16] CalculateNormalProjectionTraction (:1069-1077); the
 * traction family only at wall sites, zero elsewhere. */
static void stress_caches(double tau, double rho, const double* fpost, const double* f, int wall, const double* nor,
                          double* o) {
  double pi[3][3];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b <= a; b++) {
      pi[a][b] = 0.0;
      for (int l = 0; l < Q; l++) pi[a][b] += (fpost[l] - f[l]) * (double)CV[a][l] * (double)CV[b][l];
      pi[a][b] *= -(tau - 0.5);
    }
  for (int a = 0; a < 3; a++)
    for (int b = a + 1; b < 3; b++) pi[a][b] = pi[b][a];

  const double sxx_yy = pi[0][0] - pi[1][1], syy_zz = pi[1][1] - pi[2][2], szz_xx = pi[2][2] - pi[0][0];
  const double sxy = pi[0][1], syz = pi[1][2], szx = pi[2][0];
  const double temp1 = sxx_yy * sxx_yy + syy_zz * syy_zz + szz_xx * szz_xx;
  const double temp2 = sxy * sxy + syz * syz + szx * szx;
  o[0] = sqrt(0.5 * (temp1 + 6.0 * temp2));

  double sr = 0.0;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) sr += pi[r][c] * pi[r][c];
  sr = sqrt(sr) / (-2.0 * CS2 * rho);
  sr /= (tau - 0.5);
  o[1] = sr;

  double st[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) st[r][c] = -1.0 * pi[r][c];
  const double pressure = (rho - 1) * CS2;
  for (int r = 0; r < 3; r++) st[r][r] += -pressure;
  o[2] = st[0][0];
  o[3] = st[0][1];
  o[4] = st[0][2];
  o[5] = st[1][1];
  o[6] = st[1][2];
  o[7] = st[2][2];

  for (int k = 8; k < 17; k++) o[k] = 0.0;
  if (!wall) return;
  double t[3];
  for (int r = 0; r < 3; r++) {
    t[r] = 0.0;
    for (int c = 0; c < 3; c++) t[r] += st[r][c] * nor[c];
  }
  const double m = t[0] * nor[0] + t[1] * nor[1] + t[2] * nor[2];
  for (int k = 0; k < 3; k++) {
    o[8 + k] = t[k];
    o[11 + k] = t[k] - nor[k] * m;
    o[14 + k] = nor[k] * m;
  }
}

/* GuoZhengShiDelegate::StreamLink for wall link iPrime. Returns 0 or -1. */
static int gzs_link(const orc_sim* s, int64_t i, const hydro_t* h, int ip, double* fnew_site) {
  const orc_lattice* l = s->lat;
  const int ii = INV[ip];
  const double q = l->q[18 * i + ip - 1];
  double mw[3], fneqw[Q], fw[Q], feqw[Q], fpw[Q];
  const double fac = 1. - 1. / q;
  mw[0] = h->mx * fac;
  mw[1] = h->my * fac;
  mw[2] = h->mz * fac;
  for (int d = 0; d < Q; d++) fneqw[d] = h->fneq[d];
  if (q < 0.75) {
    if (has_iolet(l, i, ii)) {
      const int grp = l->stype[i] == 1 ? 0 : 1;
      const iolet_t* io = &s->io[grp][l->iolet_id[i]];
      if (!is_velocity_iolet(io)) {
        fnew_site[ii] = h->fpost[ip];
        return 0;
      }
      double np[3] = {(double)l->coords[3 * i] + CX[ii], (double)l->coords[3 * i + 1] + CY[ii], (double)l->coords[3 * i + 2] + CZ[ii]};
      double nv[3];
      if (iolet_velocity(io, np, (uint64_t)(unsigned int)s->t, nv)) return -1;
      for (int c = 0; c < 3; c++) {
        const double v2 = nv[c] * (q - 1) / (q + 1);
        mw[c] = q * mw[c] + (1. - q) * h->rho * v2;
      }
    } else if (has_wall(l, i, ii)) {
      fnew_site[ii] = h->fpost[ip];
      return 0;
    } else {
      const int64_t px = l->coords[3 * i] + CX[ii], py = l->coords[3 * i + 1] + CY[ii], pz = l->coords[3 * i + 2] + CZ[ii];
      const int32_t g = l->grid[(px * l->dims[1] + py) * l->dims[2] + pz];
      if (g < 0) return -2;
      const double* fn = &s->f_old[(int64_t)g * Q];
      double rn, mnx, mny, mnz, feqn[Q];
      moments(fn, &rn, &mnx, &mny, &mnz);
      const double vn[3] = {mnx / rn, mny / rn, mnz / rn};
      feq_calc(rn, mnx, mny, mnz, feqn);
      for (int c = 0; c < 3; c++) {
        const double v2 = vn[c] * (q - 1) / (q + 1);
        mw[c] = q * mw[c] + (1. - q) * h->rho * v2;
      }
      for (int d = 0; d < Q; d++) fneqw[d] = q * fneqw[d] + (1. - q) * (fn[d] - feqn[d]);
    }
  }
  feq_calc(h->rho, mw[0], mw[1], mw[2], feqw);
  for (int d = 0; d < Q; d++) fw[d] = feqw[d] + fneqw[d];
  collide(s, fw, fneqw, h->tau, fpw);
  fnew_site[ii] = fpw[ii];
  return 0;
}

/* One site: collide, then stream every link through its delegate. */
static int site_update(orc_sim* s, int64_t i, int want_macro) {
  const orc_lattice* l = s->lat;
  const int64_t n = l->n;
  hydro_t h;
  memcpy(h.f, &s->f_old[i * Q], sizeof(double) * Q);
  pre_collision(s, i, &h);
  collide(s, h.f, h.fneq, h.tau, h.fpost);
  double* fn_site = &s->f_new[i * Q];
  const int ct = site_ctype(l, i);
  int rc = 0;
  s->cpl_flag[i] = 0;
  for (int d = 0; d < Q; d++) {
    const int iol = (ct >= 2) && has_iolet(l, i, d);
    const int wal = (ct == 1 || ct >= 4) && has_wall(l, i, d);
    if (iol) {
      const int grp = l->stype[i] == 1 ? 0 : 1;
      const iolet_t* io = &s->io[grp][l->iolet_id[i]];
      const int un = INV[d];
      if (un == io->dir0) {
        s->cpl_flag[i] = 1;
        s->cpl_u[3 * i] = h.ux;
        s->cpl_u[3 * i + 1] = h.uy;
        s->cpl_u[3 * i + 2] = h.uz;
      }
      if (is_velocity_iolet(io)) {
        /* Ladd: bounce-back minus 2 w rho (u_w . c)/cs^2 at the link half-way point. */
        double hw[3] = {(double)l->coords[3 * i], (double)l->coords[3 * i + 1], (double)l->coords[3 * i + 2]};
        hw[0] += 0.5 * CX[d];
        hw[1] += 0.5 * CY[d];
        hw[2] += 0.5 * CZ[d];
        double wm[3];
        if (iolet_velocity(io, hw, (uint64_t)(unsigned int)s->t, wm)) {
          rc = -1;
          wm[0] = wm[1] = wm[2] = 0.0;
        }
        wm[0] *= h.rho;
        wm[1] *= h.rho;
        wm[2] *= h.rho;
        const double corr = 2. * W[d] * (wm[0] * CX[d] + wm[1] * CY[d] + wm[2] * CZ[d]) / CS2;
        fn_site[INV[d]] = h.fpost[d] - corr;
      } else {
        /* Nash zeroth-order pressure: ghost equilibrium at the iolet density. */
        const double rb = iolet_density(io, s->t - 1);
        const double nx = (double)io->normal_f[0], ny = (double)io->normal_f[1], nz = (double)io->normal_f[2];
        const double comp = (h.mx / h.rho) * nx + (h.my / h.rho) * ny + (h.mz / h.rho) * nz;
        double gf[Q];
        feq_calc(rb, nx * comp * rb, ny * comp * rb, nz * comp * rb, gf);
        fn_site[un] = gf[un];
      }
    } else if (wal) {
      const int id = INV[d];
      if (s->p.wall == ORC_SBB) {
        fn_site[id] = h.fpost[d];
      } else if (s->p.wall == ORC_BFL) {
        const double q = l->q[18 * i + d - 1];
        if (has_wall(l, i, id) || q < 0.5) fn_site[id] = h.fpost[d];
        else fn_site[id] = (h.fpost[d] + (2.0 * q - 1) * h.fpost[id]) / (2.0 * q);
      } else {
        if (gzs_link(s, i, &h, d, fn_site)) rc = -1;
      }
    } else {
      s->f_new[l->nbr[i * Q + d]] = h.fpost[d];
    }
  }
  if (want_macro) {
    s->rho[i] = h.rho;
    s->u[3 * i] = h.ux;
    s->u[3 * i + 1] = h.uy;
    s->u[3 * i + 2] = h.uz;
    s->wss[i] = l->wall[i] ? wss_mag(h.tau, h.fpost, h.f, &l->normal[3 * i]) : NO_VALUE;
    stress_caches(h.tau, h.rho, h.fpost, h.f, l->wall[i] != 0, &l->normal[3 * i], &s->stress[17 * i]);
  }
  (void)n;
  return rc;
}

static void site_post_step(orc_sim* s, int64_t i) {
  const orc_lattice* l = s->lat;
  if (s->p.wall != ORC_BFL || !l->wall[i]) return;
  double* fn = &s->f_new[i * Q];
  for (int d = 1; d < Q; d++) {
    if (!has_wall(l, i, d)) continue;
    const int id = INV[d];
    const double q = l->q[18 * i + d - 1];
    if (!has_wall(l, i, id) && q < 0.5) fn[id] = 2.0 * q * fn[id] + (1.0 - 2.0 * q) * fn[d];
  }
}

int orc_sim_run(orc_sim* s, int64_t steps, int want_macro) {
  const orc_lattice* l = s->lat;
  const int64_t n = l->n;
  if (want_macro && !s->stress) s->stress = (double*)calloc((size_t)(17 * n + 1), sizeof(double));
#ifdef _OPENMP
  omp_set_num_threads(s->nthreads);
#endif
  for (int64_t st = 0; st < steps; st++) {
    const int macro = want_macro && st == steps - 1;
    /* BeginPhase: WK3/WK2 DoComms (self-message and flow-rate reduction on one rank). */
    for (int g = 0; g < 2; g++)
      for (int k = 0; k < s->nio[g]; k++) {
        iolet_t* io = &s->io[g][k];
        if (!is_windkessel(io)) continue;
        io->density = io->density_new;
        io->flow = io->flow_new;
        if (io->count != 0) io->flow = io->flow * io->cfg.area / (double)io->count;
        io->flow_new = 0.0;
        io->count = 0;
      }
    int rc = 0;
#pragma omp parallel for schedule(static) reduction(| : rc)
    for (int64_t i = 0; i < n; i++) rc |= site_update(s, i, macro);
    /* Ordered coupling pass: WK3 pre-stream coupling in site order. */
    for (int64_t i = 0; i < n; i++) {
      if (!s->cpl_flag[i]) continue;
      const int grp = l->stype[i] == 1 ? 0 : 1;
      iolet_t* io = &s->io[grp][l->iolet_id[i]];
      if (!is_windkessel(io)) continue;
      if (i == io->centre) {
        const double pressure = io->density * CS2;
        if (io->cfg.kind == ORC_IOLET_WK3) {
          const double Rc = io->cfg.rc, Rp = io->cfg.rp, Cp = io->cfg.cp;
          const double pn = (Rp * Cp * pressure + (Rc + Rp) * (2.0 * io->flow - io->flow_old) + Rc * Rp * Cp * (io->flow - io->flow_old)) / (1.0 + Rp * Cp);
          io->density_new = pn / CS2;
        } else {
          /* InOutLetWK2::DoPreStreamCoupling (InOutLetWK2.cc:66-82) */
          const double R0 = io->cfg.rp, C0 = io->cfg.cp;
          const double pn = R0 / (1.0 + R0 * C0) * (io->flow + C0 * pressure);
          io->density_new = pn / CS2;
        }
      }
      const double* nrm = io->cfg.normal;
      io->flow_new += s->cpl_u[3 * i] * (-nrm[0]) + s->cpl_u[3 * i + 1] * (-nrm[1]) + s->cpl_u[3 * i + 2] * (-nrm[2]);
      io->count++;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) site_post_step(s, i);
    /* Post-stream coupling at the centre site. */
    for (int g = 0; g < 2; g++)
      for (int k = 0; k < s->nio[g]; k++) {
        iolet_t* io = &s->io[g][k];
        if (!is_windkessel(io) || io->centre < 0) continue;
        if (s->cpl_flag[io->centre] && l->iolet_id[io->centre] == k && (l->stype[io->centre] == 1 ? 0 : 1) == g) {
          io->density = io->density_new;
          if (io->cfg.kind == ORC_IOLET_WK3) io->flow_old = io->flow;
        }
      }
    /* EndIteration: swap. */
    double* tmp = s->f_old;
    s->f_old = s->f_new;
    s->f_new = tmp;
    s->t++;
    if (rc) return -1;
    /* Stability: any !(f > 0) is unstable (StabilityTester.h:100-111). */
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t k = 0; k < n * Q; k++) bad |= !(s->f_old[k] > 0.0);
    if (bad) return 1;
  }
  return 0;
}
