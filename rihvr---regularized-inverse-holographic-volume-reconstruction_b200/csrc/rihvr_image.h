// Image I/O and hologram preprocessing for the command-line driver.
//
// Replaces the OpenCV calls of RIHVR's Hologram class on the reconstruction
// path: imread of 8/16-bit grayscale frames (hologram.cu:139-199), the /255
// rescale (:401-439), I/mean - 1 (:332-358), background division
// (:1365-1432), crop (:768-887), zero padding (:889-945), and imwrite of 8-bit
// TIFFs for the outputs.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace rihvr_io {

struct Image {
  int width = 0, height = 0;
  int bits = 8;                  // 8 or 16
  std::vector<float> pixels;     // row-major grayscale values as read (0..255 or 0..65535)
};

// TIFF (8/16-bit, gray or RGB, uncompressed, PackBits or LZW, horizontal
// predictor), PNG (8/16-bit gray, 8-bit RGB) and binary PGM/PNM (P5).
// Returns false with a message on error.
bool read_image(const std::string& path, Image& out, std::string& err);

// Baseline uncompressed 8-bit grayscale TIFF.
bool write_tiff8(const std::string& path, const uint8_t* pixels, int width, int height, std::string& err);

// 8-bit grayscale PNG (zlib), as cv::imwrite writes the backgrounds.
bool write_png8(const std::string& path, const uint8_t* pixels, int width, int height, std::string& err);

// OpenCV's saturate_cast<uchar>(float): round half to even, clamp to [0, 255].
uint8_t to_u8(double v);

// Reference preprocessing to the measured hologram b (height x width real).
struct Preprocess {
  bool remove_background = false;
  int roi_x = -1, roi_y = -1, roi_size = -1;                 // Hologram::crop(center, size)
  int roi_rect_x = 0, roi_rect_y = 0, roi_rect_w = 0, roi_rect_h = 0;  // Hologram::crop(roi)
  int zero_padding = 0;
};
bool preprocess(const Image& holo, const Image* bg, const Preprocess& pp, std::vector<float>& b, int& width,
                int& height, std::string& err);

// The crop of Hologram::crop (hologram.cu:768-887) on a W0 x H0 frame: the
// rectangle (roi_rect_*) when it has an area, else a square of roi_size around
// (roi_x, roi_y) moved inside the frame (and cut to the frame when larger),
// else the whole frame.  Pixels of the rectangle outside the frame read as 0.
struct CropRect {
  int x, y, w, h;
};
inline CropRect crop_rect(const Preprocess& pp, int W0, int H0) {
  CropRect r{0, 0, W0, H0};
  if (pp.roi_rect_w > 0 && pp.roi_rect_h > 0) {
    r = {pp.roi_rect_x, pp.roi_rect_y, pp.roi_rect_w, pp.roi_rect_h};
  } else if (pp.roi_size >= 1) {
    const int size = pp.roi_size;
    r = {pp.roi_x - size / 2, pp.roi_y - size / 2, size, size};
    if (r.x < 0) r.x = 0;
    if (r.y < 0) r.y = 0;
    if (r.x + size > W0) r.x = W0 - size;
    if (r.y + size > H0) r.y = H0 - size;
    if (W0 < size) r.x = 0, r.w = W0;
    if (H0 < size) r.y = 0, r.h = H0;
  }
  return r;
}

// Mean of fl(v / 255) over a frame of 8- or 16-bit samples (stored as floats),
// as the correctly rounded exact sum divided by the count: every such value is
// 0 or at least 1/255 > 2^-8, so a whole multiple of 2^-31 below 2^9, and the
// sum is exact in 128-bit integers of 2^-31.  The device path
// (rihvr_set_hologram_frame) forms the same integer sum, so both give the same
// mean bit for bit.  false when a sample is not an integer in [0, 65535].
bool exact_unit_mean(const float* v, size_t n, double* mean);
// the 128-bit sum (hi:lo, units of 2^-31) to the mean
double unit_mean_from_sum(unsigned long long lo, unsigned long long hi, size_t n);

}  // namespace rihvr_io
