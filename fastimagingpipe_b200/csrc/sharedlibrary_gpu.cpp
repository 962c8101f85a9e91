// Drop-in replacement of the reference's sharedlibrary_gpu command line
// (pipe_interface.cpp:139-189), linked against libfip_b200.so.
//
//   sharedlibrary_gpu Visreal.fits Visimag.fits B.fits V.fits \
//       Image_Size Number_of_Baselines Frequency Cell_Size Number_of_Snapshots \
//       Tile_Size Output.fits
//
// The 11-argument form is the one README.md:30 documents (Frequency is
// accepted and unused: B is already in wavelengths).  The reference's main
// reads only 10 arguments (no Frequency, pipe_interface.cpp:171-176); that
// form is accepted too and told apart by the argument count.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "fip.h"
#include "fits_io.h"

static int usage(const char* argv0) {
  std::fprintf(stderr,
               "usage: %s Visreal.fits Visimag.fits B.fits V.fits Image_Size "
               "Number_of_Baselines [Frequency] Cell_Size Number_of_Snapshots Tile_Size "
               "Output.fits\n",
               argv0);
  return 2;
}

int main(int argc, char** argv) {
  if (argc != 11 && argc != 12) return usage(argv[0]);
  const bool with_freq = argc == 12;
  FitsImage vr, vi, B, V;
  std::string err;
  const char* names[4] = {argv[1], argv[2], argv[3], argv[4]};
  FitsImage* imgs[4] = {&vr, &vi, &B, &V};
  for (int k = 0; k < 4; ++k) {
    if (!fits_read_image(names[k], *imgs[k], err)) {
      std::fprintf(stderr, "ERROR: %s\n", err.c_str());
      return 1;
    }
  }
  size_t image_size, num_baselines, num_snapshots, unit_size;
  float cell_size;
  std::string out;
  try {
    image_size = std::stoul(argv[5]);
    num_baselines = std::stoul(argv[6]);
    int a = with_freq ? 8 : 7;
    cell_size = std::stof(argv[a]);
    num_snapshots = std::stoul(argv[a + 1]);
    unit_size = std::stoul(argv[a + 2]);
    out = argv[a + 3];
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ERROR: bad numeric argument (%s)\n", e.what());
    return usage(argv[0]);
  }
  if (num_snapshots < 3) {
    std::fprintf(stderr, "ERROR: Number_of_Snapshots must be >= 3\n");
    return 1;
  }
  const size_t need_vis = num_snapshots * num_baselines;
  if (vr.data.size() < need_vis || vi.data.size() < need_vis ||
      B.data.size() < need_vis * 2 || V.data.size() < num_snapshots * 9) {
    std::fprintf(stderr,
                 "ERROR: input sizes do not cover %zu snapshots x %zu baselines "
                 "(Visreal %zu, Visimag %zu, B %zu, V %zu values)\n",
                 num_snapshots, num_baselines, vr.data.size(), vi.data.size(), B.data.size(),
                 V.data.size());
    return 1;
  }
  if (unit_size == 0 || image_size / unit_size == 0) {
    std::fprintf(stderr, "ERROR: Tile_Size must be in [1, Image_Size]\n");
    return 1;
  }
  const size_t u = image_size / unit_size;
  std::vector<float> result(u * u);
  int st = FIpipe(vr.data.data(), vi.data.data(), B.data.data(), V.data.data(), result.data(),
                  num_baselines, image_size, num_snapshots, cell_size, unit_size);
  if (st != 0) {
    std::fprintf(stderr, "ERROR: FIpipe failed: %s (%s)\n", fip_status_string(st),
                 fip_last_error());
    return 1;
  }
  if (!fits_write_image(out, result.data(), {(long)u, (long)u}, err)) {
    std::fprintf(stderr, "Error writing FITS image: %s\n", err.c_str());
    return 1;
  }
  return 0;
}
