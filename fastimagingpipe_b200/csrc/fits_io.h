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
