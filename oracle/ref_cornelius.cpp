// ref_cornelius.cpp -- test infrastructure: a C entry point around the reference's own
// cornelius (freezeout/cornelius-c++-1.3/cornelius.cpp, compiled from the reference tree by
// build_ref.py into oracle/_ref/libref_cornelius.so). Used only to check the library's
// restatement of the algorithm; nothing in the library links it.
#include "cornelius.cpp"

extern "C" int gvh_refc_find(int dim, const double *corners, const double *dx, double iso, double *centroids,
                             double *normals, int max_elements) {
  static Cornelius cor;
  static int cur_dim = 0;
  static double cur_dx[4] = {0, 0, 0, 0}, cur_iso = 0;
  bool same = cur_dim == dim && cur_iso == iso;
  for (int k = 0; k < dim; ++k) same = same && cur_dx[k] == dx[k];
  if (!same) {
    double d[4];
    for (int k = 0; k < dim; ++k) d[k] = cur_dx[k] = dx[k];
    cor.init(dim, iso, d);
    cur_dim = dim;
    cur_iso = iso;
  }
  if (dim == 2) {
    double r0[2], r1[2];
    double *c[2] = {r0, r1};
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) c[i][j] = corners[2 * i + j];
    cor.find_surface_2d(c);
  } else if (dim == 3) {
    double buf[8];
    double *rows[4];
    double **c[2] = {rows, rows + 2};
    for (int i = 0; i < 4; ++i) rows[i] = buf + 2 * i;
    for (int i = 0; i < 8; ++i) buf[i] = corners[i];
    cor.find_surface_3d(c);
  } else {
    double buf[16];
    double *r1[8];
    double **r2[4];
    double ***c[2] = {r2, r2 + 2};
    for (int i = 0; i < 8; ++i) r1[i] = buf + 2 * i;
    for (int i = 0; i < 4; ++i) r2[i] = r1 + 2 * i;
    for (int i = 0; i < 16; ++i) buf[i] = corners[i];
    cor.find_surface_4d(c);
  }
  const int n = cor.get_Nelements();
  for (int i = 0; i < n && i < max_elements; ++i)
    for (int k = 0; k < dim; ++k) {
      centroids[i * dim + k] = cor.get_centroid_elem(i, k);
      normals[i * dim + k] = cor.get_normal_elem(i, k);
    }
  return n;
}
