// create-background: the reference's background program
// (src/core/main_create_background.cu:195-274) over the C ABI.
//
//   create-background -F <file.param>
//
// With use_median_background (7006) it writes background_XXXX.png for frames
// background_start (1003) .. background_end - 3 (1004), each the median of
// five frames (median_background_calc, :103-193).  Otherwise it writes
// background.png, the mean of the frames that
// HoloSequence::useBackgroundSubtraction reads (holo_sequence.cu:309-447),
// and background_stats.txt with alpha, beta, minimum and average.  The
// frames are read here and reduced on the GPU.
#include <getopt.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rihvr.h"
#include "rihvr_image.h"

namespace {

int fail_msg(const std::string& m) {
  std::printf("%s\n", m.c_str());
  return -1;
}

// the frames as one buffer of 8-bit, 16-bit or float samples (`bits`);
// frames listed as -1 are left zero (never read by the caller)
struct Frames {
  int width = 0, height = 0, bits = 8;
  std::vector<unsigned char> data;
};

bool load_frames(const char* pattern, const std::vector<int>& ids, Frames& out, std::string& err) {
  std::vector<rihvr_io::Image> imgs(ids.size());
  int bits = 0;
  for (size_t k = 0; k < ids.size(); ++k) {
    if (ids[k] < 0) continue;
    char name[4096];
    std::snprintf(name, sizeof(name), pattern, ids[k]);
    if (!rihvr_io::read_image(name, imgs[k], err)) return false;
    if (!out.width) {
      out.width = imgs[k].width;
      out.height = imgs[k].height;
    } else if (imgs[k].width != out.width || imgs[k].height != out.height) {
      err = std::string("frame size differs: ") + name;
      return false;
    }
    bits = bits == 0 || bits == imgs[k].bits ? imgs[k].bits : 32;
  }
  out.bits = bits ? bits : 8;
  const size_t npx = (size_t)out.width * out.height, sb = out.bits / 8;
  out.data.assign(ids.size() * npx * sb, 0);
  for (size_t k = 0; k < ids.size(); ++k) {
    if (ids[k] < 0) continue;
    unsigned char* dst = out.data.data() + k * npx * sb;
    const std::vector<float>& px = imgs[k].pixels;
    for (size_t i = 0; i < npx; ++i) {
      if (out.bits == 8) dst[i] = (unsigned char)px[i];
      else if (out.bits == 16) reinterpret_cast<unsigned short*>(dst)[i] = (unsigned short)px[i];
      else reinterpret_cast<float*>(dst)[i] = px[i];
    }
    imgs[k].pixels.clear();
    imgs[k].pixels.shrink_to_fit();
  }
  return true;
}

bool write_background(const std::string& path, const float* bg, int W, int H, std::string& err) {
  // Hologram::write of a loaded frame: convertTo(CV_8U) (hologram.cu:1587-1616)
  std::vector<unsigned char> px((size_t)W * H);
  for (size_t i = 0; i < px.size(); ++i) px[i] = rihvr_io::to_u8(bg[i]);
  return rihvr_io::write_png8(path, px.data(), W, H, err);
}

}  // namespace

int main(int argc, char** argv) {
  std::printf("Begining background calculation\n");
  std::string param_file;
  int c;
  while ((c = getopt(argc, argv, "F:")) != -1) {
    if (c == 'F') param_file = optarg;
    else return std::printf("Unknown input argument\n"), -1;
  }
  if (param_file.empty()) return std::printf("User must give input parameter file using -F flag\n"), -1;
  rihvr_params p;
  rihvr_params_default(&p);
  rihvr_file_params files;
  int rc = rihvr_read_param_file(param_file.c_str(), &p, &files);
  if (rc != RIHVR_OK) return fail_msg("reading " + param_file + ": " + rihvr_status_string(rc));
  const std::string out = files.output_path;
  std::string err;
  Frames fr;

  if (files.use_median_background) {
    const int n = files.background_end - files.background_start;
    if (files.background_start < 0 || n < 5) return fail_msg("Median background calculation requires at least 5 frames");
    std::vector<int> sel((size_t)5 * (n - 2));
    if (rihvr_background_median5_frames(n, sel.data()) != RIHVR_OK) return fail_msg(rihvr_last_error());
    std::vector<int> ids(n, -1);  // read only the frames the five-frame stack takes in
    for (int k : sel) ids[k] = files.background_start + k;
    if (!load_frames(files.image_filename, ids, fr, err)) return fail_msg(err);
    const size_t npx = (size_t)fr.width * fr.height;
    std::vector<float> bgs(npx * (n - 2));
    if (rihvr_background_median5(fr.data.data(), fr.bits, fr.width, fr.height, n, 0, bgs.data()) != RIHVR_OK)
      return fail_msg(rihvr_last_error());
    for (int j = 0; j < n - 2; ++j) {
      char name[4096];
      std::snprintf(name, sizeof(name), "%s/background_%04d.png", out.c_str(), files.background_start + j);
      if (!write_background(name, bgs.data() + (size_t)j * npx, fr.width, fr.height, err)) return fail_msg(err);
    }
    return 0;
  }

  // the frames HoloSequence reads (holo_sequence.cu:321-358 with every
  // selected frame in one chunk): start_image and image_count, or
  // background_start .. background_end - 2 when both are set; above 500
  // frames only every (count / 200)-th
  int start = files.start_image, total = files.image_count;
  if (files.background_start >= 0 && files.background_end >= 0) {
    start = files.background_start;
    total = files.background_end - files.background_start - 1;
  }
  const int step = total > 500 ? total / 200 : 1;
  const int count = total / step;
  if (count < 1) return fail_msg("no frames selected for the background");
  std::vector<int> ids(count);
  for (int k = 0; k < count; ++k) ids[k] = start + k * step;
  if (!load_frames(files.image_filename, ids, fr, err)) return fail_msg(err);
  std::vector<float> bg((size_t)fr.width * fr.height);
  double stats[4];
  if (rihvr_background_mean(fr.data.data(), fr.bits, fr.width, fr.height, count, 0, bg.data(), stats) != RIHVR_OK)
    return fail_msg(rihvr_last_error());
  std::printf("Used %d images for background calculation\n  stepsize = %d\n", count, step);
  if (!write_background(out + "/background.png", bg.data(), fr.width, fr.height, err)) return fail_msg(err);
  const std::string sf = out + "/background_stats.txt";
  FILE* f = std::fopen(sf.c_str(), "w");
  if (!f) return fail_msg("Unable to open output file: " + sf);
  for (double v : stats) std::fprintf(f, "%f\n", v);
  std::fclose(f);
  return 0;
}
