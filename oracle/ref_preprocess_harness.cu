// Test harness around the reference's own GPU preprocessing.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The
// reference's SVDPreprocessKernels.cu is compiled unmodified from where it
// lies (the path comes in as FIP_REFERENCE_PRE_CU from oracle/Makefile; it
// includes its SVDPreprocessGpu.h beside it) and this file adds one C entry
// point over its public functions (SVDPreprocessGpu.h):
//   ref_preprocess  preprocess_measurement_set_gpu + download_preprocess_outputs
//                   on host arrays: uvw [rows][3] in metres, frequencies
//                   [chans] in Hz, the two polarisations, flags and weights
//                   [rows * chans] (sample row + chan * rows), out: B
//                   [samples][2], V [9], the collapsed visibilities.
// Returns 0, or 1 when the reference throws (its message on stderr).
#include FIP_REFERENCE_PRE_CU

#include <cstdio>
#include <exception>

extern "C" int ref_preprocess(size_t rows, size_t chans, const float* uvw, const float* freqs,
                              const float* v0r, const float* v0i, const float* v3r,
                              const float* v3i, const unsigned char* f0, const unsigned char* f3,
                              const float* w0, const float* w3, float* B_out, float* V_out,
                              float* vr_out, float* vi_out) {
  try {
    const size_t ns = rows * chans;
    HostMeasurementSetData in;
    in.num_rows = rows;
    in.num_channels = chans;
    in.num_samples = ns;
    in.uvw.assign(uvw, uvw + 3 * rows);
    in.frequencies_hz.assign(freqs, freqs + chans);
    in.vis0_real.assign(v0r, v0r + ns);
    in.vis0_imag.assign(v0i, v0i + ns);
    in.vis3_real.assign(v3r, v3r + ns);
    in.vis3_imag.assign(v3i, v3i + ns);
    in.flag0.assign(f0, f0 + ns);
    in.flag3.assign(f3, f3 + ns);
    in.weight0.assign(w0, w0 + ns);
    in.weight3.assign(w3, w3 + ns);
    DevicePreprocessBuffers dev;
    preprocess_measurement_set_gpu(in, dev);
    HostPreprocessOutputs out;
    download_preprocess_outputs(dev, out);
    free_device_preprocess_buffers(dev);
    for (size_t k = 0; k < 2 * ns; ++k) B_out[k] = out.bin[k];
    for (size_t k = 0; k < 9; ++k) V_out[k] = out.vin[k];
    for (size_t k = 0; k < ns; ++k) {
      vr_out[k] = out.vis_real[k];
      vi_out[k] = out.vis_imag[k];
    }
    return 0;
  } catch (const std::exception& e) {
    fprintf(stderr, "ref_preprocess: %s\n", e.what());
    return 1;
  }
}
