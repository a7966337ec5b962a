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
// predictor) and binary PGM/PNM (P5).  Returns false with a message on error.
bool read_image(const std::string& path, Image& out, std::string& err);

// Baseline uncompressed 8-bit grayscale TIFF.
bool write_tiff8(const std::string& path, const uint8_t* pixels, int width, int height, std::string& err);

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

}  // namespace rihvr_io
