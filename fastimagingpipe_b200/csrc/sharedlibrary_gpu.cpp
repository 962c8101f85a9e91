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
//
// Two additions, neither in the reference's command line:
//
//   sharedlibrary_gpu --combined input.fits Image_Size [Frequency] Cell_Size \
//       Tile_Size Output.fits
//
// reads the preprocessing tool's combined file (svd_preprocess_gpu
// --combined-output, SVDPreprocessMain.cpp:182-258: extensions
// "TRANSFORMATION MATRICES", "VISIBILITIES", "R-COORDINATES"); the number of
// baselines is its samples per snapshot (zero-padded snapshots count their
// padding, SVDPreprocessMain.cpp:260-287) and the number of snapshots its
// third axis.  Either form takes, after its positional arguments,
//
//   --locations locations.fits [--threshold T] [--max-locations K]
//
// which also writes the transient locations of the tLISI matrix
// (fip_locate_transients: tiles below T, default 0.99, that are the minimum
// of their 3 x 3 neighbourhood) as a FITS binary table.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fip.h"
#include "fits_io.h"

static int usage(const char* argv0) {
  std::fprintf(stderr,
               "usage: %s Visreal.fits Visimag.fits B.fits V.fits Image_Size "
               "Number_of_Baselines [Frequency] Cell_Size Number_of_Snapshots Tile_Size "
               "Output.fits [--locations FILE [--threshold T] [--max-locations K]]\n"
               "       %s --combined input.fits Image_Size [Frequency] Cell_Size Tile_Size "
               "Output.fits [--locations FILE [--threshold T] [--max-locations K]]\n",
               argv0, argv0);
  return 2;
}

// Locations of the tLISI matrix `result` (host) as a FITS table.
static int write_locations(const std::string& path, const std::vector<float>& result,
                           size_t image_size, size_t unit_size, float cell, float threshold,
                           size_t max_out) {
  float* d = nullptr;
  cudaError_t e = cudaMalloc((void**)&d, result.size() * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemcpy(d, result.data(), result.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ERROR: %s\n", cudaGetErrorString(e));
    if (d) cudaFree(d);
    return 1;
  }
  std::vector<fip_location> loc(max_out);
  size_t found = 0;
  const int st = fip_locate_transients(d, image_size, unit_size, cell, threshold, loc.data(),
                                       max_out, &found, nullptr);
  cudaFree(d);
  if (st != 0) {
    std::fprintf(stderr, "ERROR: fip_locate_transients failed: %s (%s)\n",
                 fip_status_string(st), fip_last_error());
    return 1;
  }
  const size_t n = found < max_out ? found : max_out;
  std::vector<int32_t> tr(n), tc(n);
  std::vector<float> tl(n), row(n), col(n), x(n), y(n);
  for (size_t k = 0; k < n; ++k) {
    tr[k] = loc[k].tile_row;
    tc[k] = loc[k].tile_col;
    tl[k] = loc[k].tlisi;
    row[k] = loc[k].row;
    col[k] = loc[k].col;
    x[k] = loc[k].x;
    y[k] = loc[k].y;
  }
  std::string err;
  if (!fits_write_table(path,
                        {{"TILE_ROW", 'J', tr.data()}, {"TILE_COL", 'J', tc.data()},
                         {"TLISI", 'E', tl.data()}, {"ROW", 'E', row.data()},
                         {"COL", 'E', col.data()}, {"X_RAD", 'E', x.data()},
                         {"Y_RAD", 'E', y.data()}},
                        n, "LOCATIONS", err)) {
    std::fprintf(stderr, "Error writing FITS table: %s\n", err.c_str());
    return 1;
  }
  std::printf("%zu transient location(s) below tLISI %g written to %s\n", found, threshold,
              path.c_str());
  return 0;
}

int main(int argc, char** argv) {
  // Trailing options after the positional arguments.
  std::string loc_path;
  float threshold = 0.99f;
  size_t max_locations = 1024;
  std::vector<const char*> pos;
  bool combined = false;
  for (int k = 1; k < argc; ++k) {
    const std::string a = argv[k];
    if (a == "--combined" && k == 1) {
      combined = true;
    } else if (a == "--locations" || a == "--threshold" || a == "--max-locations") {
      if (k + 1 >= argc) return usage(argv[0]);
      const char* v = argv[++k];
      try {
        if (a == "--locations") loc_path = v;
        else if (a == "--threshold") threshold = std::stof(v);
        else max_locations = std::stoul(v);
      } catch (const std::exception&) {
        return usage(argv[0]);
      }
    } else {
      pos.push_back(argv[k]);
    }
  }
  size_t image_size, num_baselines, num_snapshots, unit_size;
  float cell_size;
  std::string out, err;
  std::vector<float> vis_re, vis_im, Bv, Vv;
  if (combined) {
    if (pos.size() != 5 && pos.size() != 6) return usage(argv[0]);
    CombinedInput in;
    if (!fits_read_combined(pos[0], in, err)) {
      std::fprintf(stderr, "ERROR: %s\n", err.c_str());
      return 1;
    }
    try {
      image_size = std::stoul(pos[1]);
      const size_t a = pos.size() == 6 ? 3 : 2;
      cell_size = std::stof(pos[a]);
      unit_size = std::stoul(pos[a + 1]);
      out = pos[a + 2];
    } catch (const std::exception& e) {
      std::fprintf(stderr, "ERROR: bad numeric argument (%s)\n", e.what());
      return usage(argv[0]);
    }
    num_baselines = in.samples;
    num_snapshots = in.snapshots;
    vis_re = std::move(in.vis_re);
    vis_im = std::move(in.vis_im);
    Bv = std::move(in.B);
    Vv = std::move(in.V);
  } else {
    if (pos.size() != 10 && pos.size() != 11) return usage(argv[0]);
    const bool with_freq = pos.size() == 11;
    FitsImage imgs[4];
    for (int k = 0; k < 4; ++k) {
      if (!fits_read_image(pos[k], imgs[k], err)) {
        std::fprintf(stderr, "ERROR: %s\n", err.c_str());
        return 1;
      }
    }
    try {
      image_size = std::stoul(pos[4]);
      num_baselines = std::stoul(pos[5]);
      const int a = with_freq ? 7 : 6;
      cell_size = std::stof(pos[a]);
      num_snapshots = std::stoul(pos[a + 1]);
      unit_size = std::stoul(pos[a + 2]);
      out = pos[a + 3];
    } catch (const std::exception& e) {
      std::fprintf(stderr, "ERROR: bad numeric argument (%s)\n", e.what());
      return usage(argv[0]);
    }
    vis_re = std::move(imgs[0].data);
    vis_im = std::move(imgs[1].data);
    Bv = std::move(imgs[2].data);
    Vv = std::move(imgs[3].data);
  }
  if (num_snapshots < 3) {
    std::fprintf(stderr, "ERROR: Number_of_Snapshots must be >= 3\n");
    return 1;
  }
  const size_t need_vis = num_snapshots * num_baselines;
  if (vis_re.size() < need_vis || vis_im.size() < need_vis || Bv.size() < need_vis * 2 ||
      Vv.size() < num_snapshots * 9) {
    std::fprintf(stderr,
                 "ERROR: input sizes do not cover %zu snapshots x %zu baselines "
                 "(Visreal %zu, Visimag %zu, B %zu, V %zu values)\n",
                 num_snapshots, num_baselines, vis_re.size(), vis_im.size(), Bv.size(),
                 Vv.size());
    return 1;
  }
  if (unit_size == 0 || image_size / unit_size == 0) {
    std::fprintf(stderr, "ERROR: Tile_Size must be in [1, Image_Size]\n");
    return 1;
  }
  const size_t u = image_size / unit_size;
  std::vector<float> result(u * u);
  int st = FIpipe(vis_re.data(), vis_im.data(), Bv.data(), Vv.data(), result.data(),
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
  if (!loc_path.empty())
    return write_locations(loc_path, result, image_size, unit_size, cell_size, threshold,
                           max_locations);
  return 0;
}
