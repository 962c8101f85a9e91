// Minimal FITS image reader/writer (FITS Standard 4.0, primary and IMAGE
// extension HDUs), written for the drop-in command line: the reference links
// cfitsio for read_fits_image / write_fits_image (pipe_interface.cpp:12-137),
// which is not needed for 1-D/2-D float images.
#pragma once

#include <string>
#include <vector>

struct FitsImage {
  std::vector<long> naxes;   // NAXIS1 (fastest) first
  std::vector<float> data;   // converted to float, BSCALE/BZERO applied
  std::string extname;
};

// Reads every image HDU of a file (HDUs without data are kept with empty
// data).  Returns false and sets err on failure.
bool fits_read_all(const std::string& path, std::vector<FitsImage>& hdus, std::string& err);

// Reads the first HDU with data, accepting 1-D or 2-D images like the
// reference's read_fits_image (pipe_interface.cpp:32-62).
bool fits_read_image(const std::string& path, FitsImage& img, std::string& err);

// Writes a FLOAT_IMG (BITPIX -32) primary image, replacing an existing file
// (pipe_interface.cpp:98-137).
bool fits_write_image(const std::string& path, const float* data, const std::vector<long>& naxes,
                      std::string& err);

// One column of a binary table: 'J' (int32) or 'E' (float32), nrows values.
struct FitsColumn {
  std::string name;
  char form;
  const void* data;
};

// Writes an empty primary HDU and one BINTABLE extension named `extname`,
// replacing an existing file.
bool fits_write_table(const std::string& path, const std::vector<FitsColumn>& cols, size_t nrows,
                      const std::string& extname, std::string& err);

// The preprocessing tool's combined input file (write_combined_input_fits,
// SVDPreprocessMain.cpp:182-258): IMAGE extensions "TRANSFORMATION MATRICES"
// [S][3][3], "VISIBILITIES" [S][samples][2] (real, imaginary) and
// "R-COORDINATES" [S][samples][2], found by EXTNAME.  Returned in FIpipe's
// snapshot-concatenated layout; snapshots shorter than `samples` arrive
// zero-padded (SVDPreprocessMain.cpp:260-287) and the padding counts in nb.
struct CombinedInput {
  std::vector<float> vis_re, vis_im, B, V;
  size_t samples = 0, snapshots = 0;
};
bool fits_read_combined(const std::string& path, CombinedInput& in, std::string& err);
