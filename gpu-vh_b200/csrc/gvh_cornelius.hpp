// gvh_cornelius.hpp -- iso-surface elements of one 2-, 3- or 4-cube, on the host.
//
// This is the algorithm of P. Huovinen and H. Petersen, "Particlization in hybrid models",
// Eur. Phys. J. A 48 (2012) 171, arXiv:1206.3371 ("cornelius"), which the reference ships as
// freezeout/cornelius-c++-1.3/cornelius.cpp and calls from HydroPlugin.cpp:304-305. It is
// restated here as fixed-size, allocation-free code so that many host threads can run it on
// the hypercubes the device has marked. For the freeze-out surface to be the same as the
// reference's, every decision of the published algorithm is taken the same way:
//
//  * a corner is "high" when its value >= the iso-value; a square edge is cut when its two
//    ends differ in that predicate, at the linear-interpolation point, or 1e-9 of the edge
//    length in from a corner that equals the iso-value (cornelius.cpp:1216-1283);
//  * a square with four cuts is resolved by the mean of its corners (cornelius.cpp:1297-1343);
//    each segment carries a point on the low side, which orients every normal;
//  * the squares of a cube, and the cubes of a hypercube, are visited in the order
//    (constant axis ascending, lower face first) of cornelius.cpp:1470-1510 and 1806-1845;
//  * in an ambiguous cube (an ambiguous square, or 6 segments) segments are chained into
//    polygons by matching end points within 1e-10 (L1), flipping a segment whose end matches;
//    in an ambiguous hypercube (an ambiguous cube, or 24 segments with 2 or 14 low corners)
//    polygons are grouped into polyhedra by shared segment end points;
//  * centroids are area- (volume-) weighted means of the triangles (tetrahedra) that each
//    segment spans with the element's mean point; normals are sums of the triangle
//    (tetrahedron) normals, each turned towards its segment's low-side point.
//
// The arithmetic keeps the operation order of the published implementation, so for the
// same corner values the centroids and normals agree with it to the last bit wherever the
// host's libm agrees (pow and sqrt).
#pragma once

#include <math.h>

// Host and device: the same code runs in the host pool (gvh_surface_host.cpp) and in the
// device row kernel (gvh_surface_rows.cu, compiled without FMA contraction).
#ifdef __CUDACC__
#define GVH_HD __host__ __device__
#else
#define GVH_HD
#endif

namespace gvh {
namespace iso {

constexpr int kDim = 4;
constexpr double kSameTol = 1e-10;   // end points closer than this (sum of |differences|) coincide
constexpr double kTouch = 1e-9;      // a corner on the iso-value cuts its edge this far in
constexpr int kMaxSegsPerCube = 12;
constexpr int kMaxPolysPerCube = 8;
constexpr int kMaxPolysPerHcube = 8 * kMaxPolysPerCube;
constexpr int kMaxSegsPerPoly = kMaxSegsPerCube;
constexpr int kMaxPolyhedra = 10;
constexpr int kMaxElements = 10;

enum : int { OK = 0, ERR_ODD_CUTS = -1, ERR_SHORT_POLYGON = -2, ERR_OVERFLOW = -3 };

// One piece of the surface inside a square: a segment with a point on its low side.
struct Segment {
  double p[2][kDim];
  double out[kDim];
  int s;  // which of p[] is the start; flipping the segment swaps start and end
  GVH_HD const double *start() const { return p[s]; }
  GVH_HD const double *end() const { return p[1 - s]; }
  GVH_HD void flip() { s = 1 - s; }
};

// A chain of segments of one cube, as indices into that cube's segment array.
struct Polygon {
  unsigned char seg[kMaxSegsPerPoly];
  unsigned char n;
  unsigned char ax[3];  // the cube's free axes, ascending
  unsigned char cax;    // the cube's constant axis
  bool has_centroid;
  double centroid[kDim];
};

// A group of polygons of one hypercube, as indices into the hypercube's polygon list.
struct Polyhedron {
  unsigned char poly[kMaxPolysPerHcube];
  int n;
  int ntet;
};

struct Result {
  int n;
  double centroid[kMaxElements][kDim];
  double normal[kMaxElements][kDim];
};

// The published code's pow(x, 2.0): the host compiler folds that call into this product
// (the square is exact to rounding either way), which is what its builds compute.
GVH_HD inline double sq(double x) { return x * x; }

GVH_HD inline void orient(double *nrm, const double *outp, const double *c) {
  double dot = 0;
  for (int k = 0; k < kDim; ++k) dot += (outp[k] - c[k]) * nrm[k];
  if (dot < 0)
    for (int k = 0; k < kDim; ++k) nrm[k] = -nrm[k];
}

// ---- squares -------------------------------------------------------------------------

// Segments of the square whose corner values are v[i][j] (i along free axis a, j along free
// axis b, a < b); the constant axes c0, c1 sit at values w0, w1. Returns the number of
// segments (0..2) or an error; *amb is set when the square had four cuts.
GVH_HD inline int square_segments(const double v[2][2], int c0, double w0, int c1, double w1, const double *dx,
                           double iso, Segment *seg, bool *amb) {
  *amb = false;
  const int high = (v[0][0] >= iso) + (v[0][1] >= iso) + (v[1][0] >= iso) + (v[1][1] >= iso);
  if (high == 0 || high == 4) return 0;
  int a = -1, b = -1;
  for (int k = 0; k < kDim; ++k)
    if (k != c0 && k != c1) {
      if (a < 0) a = k;
      else b = k;
    }
  const double La = dx[a], Lb = dx[b];
  double cut[4][2];
  int nc = 0;
  // position of the cut on an edge from value va (at 0) to vb (at L), or -1 if none
  auto edge = [iso](double va, double vb, double L, double *pos) -> bool {
    if ((va - iso) * (vb - iso) < 0) { *pos = (va - iso) / (va - vb) * L; return true; }
    if (va == iso && vb < iso) { *pos = kTouch * L; return true; }
    if (vb == iso && va < iso) { *pos = (1.0 - kTouch) * L; return true; }
    return false;
  };
  double pos;
  // the four edges: b = 0 along a; a = 0 along b; a = La along b; b = Lb along a
  if (edge(v[0][0], v[1][0], La, &pos)) { cut[nc][0] = pos; cut[nc][1] = 0; ++nc; }
  if (edge(v[0][0], v[0][1], Lb, &pos)) { cut[nc][0] = 0; cut[nc][1] = pos; ++nc; }
  if (edge(v[1][0], v[1][1], Lb, &pos)) { cut[nc][0] = La; cut[nc][1] = pos; ++nc; }
  if (edge(v[0][1], v[1][1], La, &pos)) { cut[nc][0] = pos; cut[nc][1] = Lb; ++nc; }
  if (nc != 2 && nc != 4) return nc == 0 ? 0 : ERR_ODD_CUTS;

  double outp[2][2];
  if (nc == 4) {
    *amb = true;
    double mid = 0;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) mid += 0.25 * v[i][j];
    // cuts pair up (0,1)(2,3) unless the centre and the (0,0) corner are on the same side
    if ((v[0][0] < iso && mid < iso) || (v[0][0] > iso && mid > iso))
      for (int k = 0; k < 2; ++k) {
        const double t = cut[1][k];
        cut[1][k] = cut[2][k];
        cut[2][k] = t;
      }
    if (mid - iso < 0) {
      outp[0][0] = outp[1][0] = 0.5 * La;
      outp[0][1] = outp[1][1] = 0.5 * Lb;
    } else if (v[0][0] - iso < 0) {
      outp[0][0] = 0; outp[0][1] = 0;
      outp[1][0] = La; outp[1][1] = Lb;
    } else {
      outp[0][0] = La; outp[0][1] = 0;
      outp[1][0] = 0; outp[1][1] = Lb;
    }
  } else {
    // the mean of the low corners
    double sa = 0, sb = 0;
    int nlow = 0;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        if (v[i][j] < iso) {
          sa += i * La;
          sb += j * Lb;
          ++nlow;
        }
    outp[0][0] = nlow > 0 ? sa / double(nlow) : sa;
    outp[0][1] = nlow > 0 ? sb / double(nlow) : sb;
  }
  const int nseg = nc / 2;
  for (int m = 0; m < nseg; ++m) {
    Segment &g = seg[m];
    for (int e = 0; e < 2; ++e) {
      g.p[e][a] = cut[2 * m + e][0];
      g.p[e][b] = cut[2 * m + e][1];
      g.p[e][c0] = w0;
      g.p[e][c1] = w1;
    }
    g.out[a] = outp[m][0];
    g.out[b] = outp[m][1];
    g.out[c0] = w0;
    g.out[c1] = w1;
    g.s = 0;
  }
  return nseg;
}

// Centroid and normal of a segment of a 2-cube (constant axes 0 and 1; free axes 2 and 3).
GVH_HD inline void segment_element(const Segment &g, double *centroid, double *normal) {
  const double *p0 = g.start(), *p1 = g.end(), *outp = g.out;
  for (int k = 0; k < kDim; ++k) centroid[k] = (p0[k] + p1[k]) / 2.0;
  normal[2] = -(p1[3] - p0[3]);
  normal[3] = p1[2] - p0[2];
  normal[0] = 0;
  normal[1] = 0;
  orient(normal, outp, centroid);
}

// ---- polygons ------------------------------------------------------------------------
// A polygon's segments live in its cube's segment array `segs`, which every polygon function
// takes beside the polygon.

GVH_HD inline void polygon_init(Polygon &P, int cax) {
  P.n = 0;
  P.cax = (unsigned char)cax;
  P.has_centroid = false;
  int m = 0;
  for (int k = 0; k < kDim; ++k)
    if (k != cax) P.ax[m++] = (unsigned char)k;
}

GVH_HD inline double l1_distance(const double *x, const double *y) {
  double d = 0;
  for (int k = 0; k < kDim; ++k) d += fabs(x[k] - y[k]);
  return d;
}

// Appends segment g when it continues the chain (its start or end is the last segment's end).
GVH_HD inline bool polygon_extend(Polygon &P, Segment *segs, int g) {
  if (P.n == 0) {
    P.seg[0] = (unsigned char)g;
    P.n = 1;
    return true;
  }
  const double *tail = segs[P.seg[P.n - 1]].end();
  const double *g0 = segs[g].start(), *g1 = segs[g].end();
  const double d_start = l1_distance(g0, tail);
  const double d_end = l1_distance(g1, tail);
  if (d_start < kSameTol || d_end < kSameTol) {
    if (d_end < kSameTol) segs[g].flip();
    P.seg[P.n] = (unsigned char)g;
    ++P.n;
    return true;
  }
  return false;
}

GVH_HD inline void polygon_add(Polygon &P, int g) { P.seg[P.n++] = (unsigned char)g; }

GVH_HD inline const double *polygon_centroid(Polygon &P, const Segment *segs) {
  if (P.has_centroid) return P.centroid;
  double mean[kDim] = {0, 0, 0, 0};
  for (int i = 0; i < P.n; ++i) {
    const double *p0 = segs[P.seg[i]].start(), *p1 = segs[P.seg[i]].end();
    for (int k = 0; k < kDim; ++k) mean[k] += p0[k] + p1[k];
  }
  for (int k = 0; k < kDim; ++k) mean[k] = mean[k] / double(2.0 * P.n);
  if (P.n == 3) {
    for (int k = 0; k < kDim; ++k) P.centroid[k] = mean[k];
    P.has_centroid = true;
    return P.centroid;
  }
  const int x = P.ax[0], y = P.ax[1], z = P.ax[2];
  double wsum[kDim] = {0, 0, 0, 0};
  double area = 0;
  for (int i = 0; i < P.n; ++i) {
    const double *p0 = segs[P.seg[i]].start(), *p1 = segs[P.seg[i]].end();
    double cm[kDim], u[kDim], w[kDim];
    for (int k = 0; k < kDim; ++k) cm[k] = (p0[k] + p1[k] + mean[k]) / 3.0;
    for (int k = 0; k < kDim; ++k) {
      u[k] = p0[k] - mean[k];
      w[k] = p1[k] - mean[k];
    }
    const double A = 0.5 * sqrt(sq(u[y] * w[z] - u[z] * w[y]) + sq(u[x] * w[z] - u[z] * w[x]) +
                                sq(u[y] * w[x] - u[x] * w[y]));
    for (int k = 0; k < kDim; ++k) wsum[k] += cm[k] * A;
    area += A;
  }
  for (int k = 0; k < kDim; ++k) P.centroid[k] = wsum[k] / area;
  P.has_centroid = true;
  return P.centroid;
}

GVH_HD inline void polygon_normal(Polygon &P, const Segment *segs, double *normal) {
  const double *c = polygon_centroid(P, segs);
  const int x = P.ax[0], y = P.ax[1], z = P.ax[2];
  for (int k = 0; k < kDim; ++k) normal[k] = 0;
  for (int i = 0; i < P.n; ++i) {
    const double *p0 = segs[P.seg[i]].start(), *p1 = segs[P.seg[i]].end(), *outp = segs[P.seg[i]].out;
    double u[kDim], w[kDim], t[kDim];
    for (int k = 0; k < kDim; ++k) {
      u[k] = p0[k] - c[k];
      w[k] = p1[k] - c[k];
    }
    t[x] = 0.5 * (u[y] * w[z] - u[z] * w[y]);
    t[y] = -0.5 * (u[x] * w[z] - u[z] * w[x]);
    t[z] = 0.5 * (u[x] * w[y] - u[y] * w[x]);
    t[P.cax] = 0;
    orient(t, outp, c);
    for (int k = 0; k < kDim; ++k) normal[k] += t[k];
  }
}

// ---- cubes ---------------------------------------------------------------------------

struct CubeWork {
  Segment seg[kMaxSegsPerCube];
  int nseg;
  Polygon poly[kMaxPolysPerCube];
  int npoly;
  bool ambiguous;
};

// Polygons of the cube with corner values v[i][j][k] over the free axes (ascending); its
// constant axis cax sits at value w.
GVH_HD inline int cube_polygons(const double v[2][2][2], int cax, double w, const double *dx, double iso, CubeWork &cw) {
  int fa[3], m = 0;
  for (int k = 0; k < kDim; ++k)
    if (k != cax) fa[m++] = k;
  cw.nseg = 0;
  cw.npoly = 0;
  int amb_squares = 0;
  for (int f = 0; f < 3; ++f) {  // the free axis held fixed by the square
    const int ax = fa[f];
    for (int side = 0; side < 2; ++side) {
      double sq[2][2];
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) sq[i][j] = f == 0 ? v[side][i][j] : f == 1 ? v[i][side][j] : v[i][j][side];
      bool amb = false;
      const int ns = square_segments(sq, cax, w, ax, side * dx[ax], dx, iso, cw.seg + cw.nseg, &amb);
      if (ns < 0) return ns;
      cw.nseg += ns;
      amb_squares += amb;
    }
  }
  cw.ambiguous = amb_squares > 0 || cw.nseg == 6;
  if (cw.nseg == 0) return OK;
  if (!cw.ambiguous) {
    polygon_init(cw.poly[0], cax);
    for (int i = 0; i < cw.nseg; ++i) polygon_add(cw.poly[0], i);
    cw.npoly = 1;
    return OK;
  }
  bool used[kMaxSegsPerCube] = {};
  int nused = 0;
  while (nused < cw.nseg) {
    if (cw.nseg - nused < 3) return ERR_SHORT_POLYGON;
    if (cw.npoly == kMaxPolysPerCube) return ERR_OVERFLOW;
    Polygon &P = cw.poly[cw.npoly];
    polygon_init(P, cax);
    // scan for a segment that continues the chain; after each addition scan again from the
    // second segment (the first one is always in the first polygon)
    int i = 0;
    while (i < cw.nseg) {
      if (!used[i] && polygon_extend(P, cw.seg, i)) {
        used[i] = true;
        ++nused;
        i = 1;
        continue;
      }
      ++i;
    }
    ++cw.npoly;
  }
  return OK;
}

// ---- polyhedra -----------------------------------------------------------------------

struct HypercubeWork {
  CubeWork cube[8];
  // the hypercube's polygons in the order they were found: cube, then index in that cube
  unsigned char pcube[kMaxPolysPerHcube], pidx[kMaxPolysPerHcube];
  Polyhedron hedra[kMaxPolyhedra];
  GVH_HD Polygon &polygon(int q) { return cube[pcube[q]].poly[pidx[q]]; }
  GVH_HD Segment *segments(int q) { return cube[pcube[q]].seg; }
};

// Segments l (of the new polygon) and m (already in the polyhedron) share a point: m's start
// is one of l's end points.
GVH_HD inline bool segments_touch(const Segment &l, const Segment &m) {
  const double *l0 = l.start(), *l1 = l.end(), *m0 = m.start();
  double d0 = 0, d1 = 0;
  for (int k = 0; k < kDim; ++k) {
    d0 += fabs(l0[k] - m0[k]);
    d1 += fabs(l1[k] - m0[k]);
    if (d0 > kSameTol && d1 > kSameTol) return false;
  }
  return true;
}

// Adds the hypercube's polygon q to H when H is empty or q shares a point with one of H's
// polygons.
GVH_HD inline bool polyhedron_extend(Polyhedron &H, HypercubeWork &hw, int q) {
  const Polygon &P = hw.polygon(q);
  if (H.n == 0) {
    H.poly[0] = (unsigned char)q;
    H.n = 1;
    H.ntet = P.n;
    return true;
  }
  const Segment *ps = hw.segments(q);
  for (int i = 0; i < H.n; ++i) {
    const Polygon &Q = hw.polygon(H.poly[i]);
    const Segment *qs = hw.segments(H.poly[i]);
    for (int j = 0; j < P.n; ++j)
      for (int k = 0; k < Q.n; ++k)
        if (segments_touch(ps[P.seg[j]], qs[Q.seg[k]])) {
          H.poly[H.n++] = (unsigned char)q;
          H.ntet += P.n;
          return true;
        }
  }
  return false;
}

// The 3-volume normal (a x b x c)/6 of the tetrahedron spanned by a, b, c.
GVH_HD inline void tetra_normal(const double *a, const double *b, const double *c, double *n) {
  const double bc01 = b[0] * c[1] - b[1] * c[0];
  const double bc02 = b[0] * c[2] - b[2] * c[0];
  const double bc03 = b[0] * c[3] - b[3] * c[0];
  const double bc12 = b[1] * c[2] - b[2] * c[1];
  const double bc13 = b[1] * c[3] - b[3] * c[1];
  const double bc23 = b[2] * c[3] - b[3] * c[2];
  n[0] = 1.0 / 6.0 * (a[1] * bc23 - a[2] * bc13 + a[3] * bc12);
  n[1] = -1.0 / 6.0 * (a[0] * bc23 - a[2] * bc03 + a[3] * bc02);
  n[2] = 1.0 / 6.0 * (a[0] * bc13 - a[1] * bc03 + a[3] * bc01);
  n[3] = -1.0 / 6.0 * (a[0] * bc12 - a[1] * bc02 + a[2] * bc01);
}

GVH_HD inline void polyhedron_element(const Polyhedron &H, HypercubeWork &hw, double *centroid, double *normal) {
  double mean[kDim] = {0, 0, 0, 0};
  for (int i = 0; i < H.n; ++i) {
    const Polygon &P = hw.polygon(H.poly[i]);
    const Segment *ps = hw.segments(H.poly[i]);
    for (int j = 0; j < P.n; ++j) {
      const double *p0 = ps[P.seg[j]].start(), *p1 = ps[P.seg[j]].end();
      for (int k = 0; k < kDim; ++k) mean[k] += p0[k] + p1[k];
    }
  }
  for (int k = 0; k < kDim; ++k) mean[k] = mean[k] / double(2.0 * H.ntet);
  double wsum[kDim] = {0, 0, 0, 0};
  double vol = 0;
  for (int i = 0; i < H.n; ++i) {
    Polygon &P = hw.polygon(H.poly[i]);
    const Segment *ps = hw.segments(H.poly[i]);
    const double *pc = polygon_centroid(P, ps);
    for (int j = 0; j < P.n; ++j) {
      const double *p0 = ps[P.seg[j]].start(), *p1 = ps[P.seg[j]].end();
      double cm[kDim], a[kDim], b[kDim], c[kDim], n[kDim];
      for (int k = 0; k < kDim; ++k) cm[k] = (p0[k] + p1[k] + pc[k] + mean[k]) / 4.0;
      for (int k = 0; k < kDim; ++k) {
        a[k] = p0[k] - mean[k];
        b[k] = p1[k] - mean[k];
        c[k] = pc[k] - mean[k];
      }
      tetra_normal(a, b, c, n);
      double V = 0;
      for (int k = 0; k < kDim; ++k) V += n[k] * n[k];
      V = sqrt(V);
      for (int k = 0; k < kDim; ++k) wsum[k] += cm[k] * V;
      vol += V;
    }
  }
  for (int k = 0; k < kDim; ++k) centroid[k] = wsum[k] / vol;
  for (int k = 0; k < kDim; ++k) normal[k] = 0;
  for (int i = 0; i < H.n; ++i) {
    Polygon &P = hw.polygon(H.poly[i]);
    const Segment *ps = hw.segments(H.poly[i]);
    const double *pc = polygon_centroid(P, ps);
    for (int j = 0; j < P.n; ++j) {
      const double *p0 = ps[P.seg[j]].start(), *p1 = ps[P.seg[j]].end(), *outp = ps[P.seg[j]].out;
      double a[kDim], b[kDim], c[kDim], n[kDim];
      for (int k = 0; k < kDim; ++k) {
        a[k] = p0[k] - centroid[k];
        b[k] = p1[k] - centroid[k];
        c[k] = pc[k] - centroid[k];
      }
      tetra_normal(a, b, c, n);
      orient(n, outp, centroid);
      for (int k = 0; k < kDim; ++k) normal[k] += n[k];
    }
  }
}

// ---- the three entry points ------------------------------------------------------------

// 2-cube: corner values v[i][j] over (axis 2, axis 3) with spacings dx[2], dx[3].
GVH_HD inline int find_2d(const double v[2][2], const double *dx4, double iso, Result &r) {
  r.n = 0;
  Segment seg[2];
  bool amb;
  const int ns = square_segments(v, 0, 0.0, 1, 0.0, dx4, iso, seg, &amb);
  if (ns < 0) return ns;
  for (int i = 0; i < ns; ++i) segment_element(seg[i], r.centroid[i], r.normal[i]);
  r.n = ns;
  return OK;
}

// 3-cube: corner values v[i][j][k] over axes 1, 2, 3.
GVH_HD inline int find_3d(const double v[2][2][2], const double *dx4, double iso, Result &r, CubeWork &cw) {
  r.n = 0;
  int high = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) high += v[i][j][k] >= iso;
  if (high == 0 || high == 8) return OK;
  const int rc = cube_polygons(v, 0, 0.0, dx4, iso, cw);
  if (rc) return rc;
  if (cw.npoly > kMaxElements) return ERR_OVERFLOW;
  for (int i = 0; i < cw.npoly; ++i) {
    const double *c = polygon_centroid(cw.poly[i], cw.seg);
    for (int k = 0; k < kDim; ++k) r.centroid[i][k] = c[k];
    polygon_normal(cw.poly[i], cw.seg, r.normal[i]);
  }
  r.n = cw.npoly;
  return OK;
}

// 4-cube: corner values v[i][j][k][l] over axes 0..3.
GVH_HD inline int find_4d(const double v[2][2][2][2], const double *dx4, double iso, Result &r, HypercubeWork &hw) {
  r.n = 0;
  int high = 0;
  for (int i = 0; i < 16; ++i) high += (&v[0][0][0][0])[i] >= iso;
  if (high == 0 || high == 16) return OK;
  int npoly = 0, nseg = 0, amb_cubes = 0;
  for (int ax = 0; ax < kDim; ++ax)
    for (int side = 0; side < 2; ++side) {
      double cu[2][2][2];
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
          for (int k = 0; k < 2; ++k)
            cu[i][j][k] = ax == 0   ? v[side][i][j][k]
                          : ax == 1 ? v[i][side][j][k]
                          : ax == 2 ? v[i][j][side][k]
                                    : v[i][j][k][side];
      const int c = 2 * ax + side;
      CubeWork &cw = hw.cube[c];
      const int rc = cube_polygons(cu, ax, side * dx4[ax], dx4, iso, cw);
      if (rc) return rc;
      for (int p = 0; p < cw.npoly; ++p) {
        hw.pcube[npoly] = (unsigned char)c;
        hw.pidx[npoly] = (unsigned char)p;
        ++npoly;
      }
      nseg += cw.nseg;
      amb_cubes += cw.ambiguous;
    }
  bool ambiguous = amb_cubes > 0;
  if (!ambiguous) {
    int low = 16 - high;
    if (low > 8) low = 16 - low;
    ambiguous = nseg == 24 && low == 2;
  }
  int nh = 0;
  if (!ambiguous) {
    Polyhedron &H = hw.hedra[0];
    H.n = 0;
    H.ntet = 0;
    for (int p = 0; p < npoly; ++p) {
      H.poly[H.n++] = (unsigned char)p;
      H.ntet += hw.polygon(p).n;
    }
    nh = 1;
  } else {
    bool used[kMaxPolysPerHcube] = {};
    int nused = 0;
    while (nused < npoly) {
      if (nh == kMaxPolyhedra) return ERR_OVERFLOW;
      Polyhedron &H = hw.hedra[nh];
      H.n = 0;
      H.ntet = 0;
      int i = 0;
      while (i < npoly) {
        if (!used[i] && polyhedron_extend(H, hw, i)) {
          used[i] = true;
          ++nused;
          i = 1;
          continue;
        }
        ++i;
      }
      ++nh;
    }
  }
  if (nh > kMaxElements) return ERR_OVERFLOW;
  for (int h = 0; h < nh; ++h) polyhedron_element(hw.hedra[h], hw, r.centroid[h], r.normal[h]);
  r.n = nh;
  return OK;
}

}  // namespace iso
}  // namespace gvh
