// gvh-run: command-line entry mirroring the reference's executable (RunHydroWrapper.cpp:9-18,
// HydroWrapper.cpp:17-87, flags of CommandLineArguments.cpp:17-24): -c <config dir> with
// lattice/hydro/ic.properties, -o <output dir>; the initial state is read from
// <cwd>/input/*.dat (initial-condition type 10). Extra flags select the reference's
// compile-time switches: --conformal, --no-bulk, --ideal, --theta <v>, --mixed, --cartesian; --no-dump and
// --no-surface turn off the field dumps and <output dir>/surface.dat.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <string>

#include "../../include/gvh.h"

int main(int argc, char **argv) {
  std::string config = "rhic-conf", out = "output";
  gvh_options o;
  gvh_default_options(&o);
  int outputs = GVH_RUN_FIELDS | GVH_RUN_SURFACE;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if ((a == "-c" || a == "--config") && i + 1 < argc) config = argv[++i];
    else if ((a == "-o" || a == "--output") && i + 1 < argc) out = argv[++i];
    else if (a == "--conformal") o.eos = GVH_EOS_CONFORMAL;
    else if (a == "--no-bulk") o.bulk = 0;
    else if (a == "--ideal") { o.bulk = 0; o.shear = 0; }
    else if (a == "--theta" && i + 1 < argc) o.theta = atof(argv[++i]);
    else if (a == "--mixed") o.precision = GVH_PRECISION_MIXED;
    else if (a == "--cartesian") o.coordinates = GVH_COORDINATES_CARTESIAN;
    else if (a == "--no-dump") outputs &= ~GVH_RUN_FIELDS;
    else if (a == "--no-surface") outputs &= ~GVH_RUN_SURFACE;
    else if (a == "-h" || a == "-t") continue;  // the reference accepts these too
    else {
      fprintf(stderr, "usage: %s [-c config_dir] [-o output_dir] [--conformal] [--no-bulk] [--ideal] "
                      "[--theta v] [--mixed] [--cartesian] [--no-dump] [--no-surface]\n", argv[0]);
      return 2;
    }
  }
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) return 1;
  gvh_lattice_params L;
  gvh_hydro_params H;
  gvh_ic_params ic;
  if (gvh_read_lattice_parameters(config.c_str(), &L) || gvh_read_hydro_parameters(config.c_str(), &H) ||
      gvh_read_ic_parameters(config.c_str(), &ic)) {
    fprintf(stderr, "gvh-run: %s\n", gvh_plugin_last_error());
    return 1;
  }
  printf("Grid size = %d x %d x %d\n", L.numLatticePointsX, L.numLatticePointsY, L.numLatticePointsRapidity);
  printf("spatial resolution = (%.3f, %.3f, %.3f)\n", L.latticeSpacingX, L.latticeSpacingY, L.latticeSpacingRapidity);
  printf("eta/s = %.6f\n", H.shearViscosityToEntropyDensity);
  gvh_run_report r;
  int rc = gvh_run(&L, &ic, &H, cwd, out.c_str(), &o, outputs, &r);
  if (rc) {
    fprintf(stderr, "gvh-run: %s\n", gvh_plugin_last_error());
    return 1;
  }
  if (r.frozen_out) printf("\nAll cells have dropped below freezeout energy density\n");
  printf("Average time/step: %.3f ms\n", r.average_ms_per_step);
  printf("steps = %lld, tau = %.3f fm/c, status = %u\n", r.steps, r.tau_end, r.status);
  if (outputs & GVH_RUN_SURFACE)
    printf("surface elements = %lld (finder %.3f s)\n", r.surface_elements, r.surface_seconds);
  return 0;
}
