// sparse-inverse-recon: command-line driver with the reference's interface
// (src/core/main_sparse_inverse.cu:43-198): -F <file.param> [-S 0|1] [-G 0|1].
// -G 1 also runs the reference's separate segmentation program
// (src/core/main_segmentation.cu:37-138) on the final volume in device memory
// and writes centroids_XXXX.csv, centroids_weighted_XXXX.csv and
// centroids_verbose_XXXX.csv with the .param file's segment_* settings.
//
// Reads the .param file, loads and preprocesses the hologram frame, runs the
// reconstruction through the C ABI and writes the reference's output files:
// enh.tif, initial_measured.tif / estimate_initial.tif / initial_residual.tif,
// estimate_final.tif / residual_final.tif, all_metrics.csv, the plane images
// inverse_XXXX.tif (+ _phase_, _real_, _imag_) when output_planes is set, the
// max projections cmb_{xy,xz,yz}.tif and the voxel list inverse_voxels.csv.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rihvr.h"
#include "rihvr_image.h"

using rihvr_io::to_u8;

namespace {

bool fail_msg(const std::string& m) {
  std::fprintf(stderr, "%s\n", m.c_str());
  return false;
}

bool write_scaled(const std::string& path, const std::vector<float>& v, int W, int H, double lo, double hi) {
  // Hologram::write(filename, min, max) (hologram.cu:1633-1654)
  std::vector<uint8_t> px(v.size());
  const double s = 255.0 / (hi - lo);
  for (size_t i = 0; i < v.size(); ++i) px[i] = to_u8((v[i] - lo) * s);
  std::string err;
  return rihvr_io::write_tiff8(path, px.data(), W, H, err) || fail_msg(err);
}

bool write_minmax(const std::string& path, const std::vector<float>& v, int W, int H) {
  // Hologram::write(filename) for a non-loaded state: min-max to 0..255 (:1587-1616)
  const auto mm = std::minmax_element(v.begin(), v.end());
  const double lo = *mm.first, hi = *mm.second;
  if (!(hi > lo)) {
    std::vector<uint8_t> px(v.size(), 0);
    std::string err;
    return rihvr_io::write_tiff8(path, px.data(), W, H, err) || fail_msg(err);
  }
  return write_scaled(path, v, W, H, lo, hi);
}

struct Planes {
  rihvr_ctx* ctx;
  int W, H, Nz;
  std::vector<std::complex<float>> buf;
  const std::complex<float>* get(int z) {
    buf.resize((size_t)W * H);
    if (rihvr_get_plane(ctx, z, reinterpret_cast<float*>(buf.data()), 0) != RIHVR_OK) return nullptr;
    return buf.data();
  }
};

// cv::magnitude of a complex voxel, in float as OpenCV computes it
inline float magnitude(std::complex<float> v) { return std::sqrt(v.real() * v.real() + v.imag() * v.imag()); }

// cv::Mat::convertTo(CV_8U, 255) of a value already scaled to [0, 1]:
// saturate_cast<uchar>, rounding half to even
inline uint8_t u8_of_unit(float v) { return to_u8(v * 255.0f); }

// The affine map (plane - lo) / (hi - lo) that the reference writes as a
// cv::Mat expression, which OpenCV evaluates as convertTo(alpha, beta) with
// alpha = 1 / (hi - lo) and beta = -lo * alpha, in float.
struct UnitMap {
  float alpha, beta;
  UnitMap(double lo, double hi) {
    const double a = 1.0 / (hi - lo);
    alpha = (float)a;
    beta = (float)(-lo * a);
  }
  float operator()(float v) const { return v * alpha + beta; }
};

// Global magnitude range over the planes (the first loop of savePlanes,
// sparse_compressive_holo.cu:1045-1063, and of saveProjections,
// sparse_volume.cu:708-726): one pass over the volume.
bool magnitude_range(Planes& pl, double& lo, double& hi) {
  lo = hi = 0;
  for (int z = 0; z < pl.Nz; ++z) {
    const auto* p = pl.get(z);
    if (!p) return fail_msg(rihvr_last_error());
    float a = magnitude(p[0]), b = a;
    for (size_t i = 1; i < (size_t)pl.W * pl.H; ++i) {
      const float m = magnitude(p[i]);
      a = std::min(a, m);
      b = std::max(b, m);
    }
    if (z == 0) { lo = a; hi = b; }
    lo = std::min(lo, (double)a);
    hi = std::max(hi, (double)b);
  }
  return true;
}

// The reference's three volume writers in one further pass over the planes:
// * SparseCompressiveHolo::savePlanes (sparse_compressive_holo.cu:1039-1194):
//   prefix_XXXX.tif magnitude over the global range, prefix_phase_XXXX.tif
//   phase in [0, 2 pi) over 2 pi, prefix_real/imag_XXXX.tif over
//   +-sqrt(global max) / 10 (when planes_prefix is not empty);
// * SparseVolume::saveProjections, MAX_CMB (sparse_volume.cu:684-813):
//   cmb_xy/xz/yz.tif maxima of the scaled magnitude; the XY projection starts
//   from zeros and folds in planes z > 0 only, as the reference does;
// * SparseVolume::saveData (sparse_volume.cu:518-560): inverse_voxels.csv,
//   the non-zero voxels with their intensity, plane by plane in raster order.
bool save_volume_outputs(Planes& pl, const std::string& planes_prefix, const std::string& output_path,
                         const std::string& cmb_prefix, const std::string& sparse_prefix) {
  double gmin, gmax;
  if (!magnitude_range(pl, gmin, gmax)) return false;
  const int W = pl.W, H = pl.H, Z = pl.Nz;
  const size_t n = (size_t)W * H;
  const UnitMap mag_map(gmin, gmax);
  const double rmax = std::sqrt(gmax) / 10.0;
  const UnitMap ri_map(-rmax, rmax);
  std::vector<uint8_t> px(n);
  std::vector<float> xy(n, 0.f), xz((size_t)Z * W, 0.f), yz((size_t)H * Z, 0.f), colmax(W);
  std::string err;
  char name[4096];
  const std::string csv = output_path + "/" + sparse_prefix + ".csv";
  FILE* f = std::fopen(csv.c_str(), "w");
  if (!f) return fail_msg("Unable to open file: " + csv);
  std::fprintf(f, "x, y, z, value\n");
  auto bail = [&](const std::string& m) {
    std::fclose(f);
    return fail_msg(m);
  };
  for (int z = 0; z < Z; ++z) {
    const auto* p = pl.get(z);
    if (!p) return bail(rihvr_last_error());
    if (!planes_prefix.empty()) {
      for (size_t i = 0; i < n; ++i) px[i] = u8_of_unit(mag_map(magnitude(p[i])));
      std::snprintf(name, sizeof(name), "%s_%04d.tif", planes_prefix.c_str(), z);
      if (!rihvr_io::write_tiff8(name, px.data(), W, H, err)) return bail(err);
      for (size_t i = 0; i < n; ++i) {
        float ph = std::atan2(p[i].imag(), p[i].real());  // cv::phase: [0, 2 pi)
        if (ph < 0) ph += (float)(2.0 * M_PI);
        px[i] = u8_of_unit(ph * (float)(1.0 / (2.0 * M_PI)));
      }
      std::snprintf(name, sizeof(name), "%s_phase_%04d.tif", planes_prefix.c_str(), z);
      if (!rihvr_io::write_tiff8(name, px.data(), W, H, err)) return bail(err);
      for (size_t i = 0; i < n; ++i) px[i] = u8_of_unit(ri_map(p[i].real()));
      std::snprintf(name, sizeof(name), "%s_real_%04d.tif", planes_prefix.c_str(), z);
      if (!rihvr_io::write_tiff8(name, px.data(), W, H, err)) return bail(err);
      for (size_t i = 0; i < n; ++i) px[i] = u8_of_unit(ri_map(p[i].imag()));
      std::snprintf(name, sizeof(name), "%s_imag_%04d.tif", planes_prefix.c_str(), z);
      if (!rihvr_io::write_tiff8(name, px.data(), W, H, err)) return bail(err);
    }
    std::fill(colmax.begin(), colmax.end(), -1e30f);
    for (int y = 0; y < H; ++y) {
      float rowmax = -1e30f;
      for (int x = 0; x < W; ++x) {
        const std::complex<float> v = p[(size_t)y * W + x];
        const float s = mag_map(magnitude(v));
        rowmax = std::max(rowmax, s);
        colmax[x] = std::max(colmax[x], s);
        if (z > 0) xy[(size_t)y * W + x] = std::max(xy[(size_t)y * W + x], s);
        if (v.real() != 0.f || v.imag() != 0.f)
          std::fprintf(f, "%d, %d, %d, %e\n", x, y, z, v.real() * v.real() + v.imag() * v.imag());
      }
      yz[(size_t)y * Z + z] = rowmax;
    }
    for (int x = 0; x < W; ++x) xz[(size_t)z * W + x] = colmax[x];
  }
  std::fclose(f);
  auto put = [&](const std::vector<float>& v, int w, int h, const std::string& tag) {
    std::vector<uint8_t> q(v.size());
    for (size_t i = 0; i < v.size(); ++i) q[i] = u8_of_unit(v[i]);
    const std::string file = output_path + cmb_prefix + "_" + tag + ".tif";  // no separator, as the reference
    return rihvr_io::write_tiff8(file, q.data(), w, h, err) || fail_msg(err);
  };
  return put(xy, W, H, "xy") && put(xz, W, Z, "xz") && put(yz, Z, H, "yz");
}

// SparseSegmentation + ObjectCloud::blobSizeFilter + writeCentroids
// (main_segmentation.cu:100-128)
bool segment_and_save(rihvr_ctx* ctx, const rihvr_file_params& files, const std::string& out) {
  rihvr_segment_params sp;
  rihvr_segment_params_default(&sp);
  sp.min_intensity = files.segment_min_intensity;
  sp.close_size = files.segment_close_size;
  sp.min_area = files.segment_min_area;
  std::vector<rihvr_object> objs(1 << 16);
  int n = 0;
  rihvr_segment_info info;
  int rc = rihvr_segment(ctx, &sp, objs.data(), (int)objs.size(), &n, &info);
  if (rc == RIHVR_ERR_INVALID_ARGUMENT && n > (int)objs.size()) {
    objs.resize(n);
    rc = rihvr_segment(ctx, &sp, objs.data(), (int)objs.size(), &n, &info);
  }
  if (rc != RIHVR_OK) return fail_msg(std::string("rihvr_segment: ") + rihvr_last_error());
  std::printf("max intensity = %f, thr = %f\n", info.max_intensity, info.threshold);
  std::printf("Number of particles: %lld\n", info.labelled_objects);
  std::printf("blobSizeFilter removed %lld objects\n", info.labelled_objects - n);
  char name[4096];
  const char* kinds[3] = {"centroids", "centroids_weighted", "centroids_verbose"};
  for (int k = 0; k < 3; ++k) {
    std::snprintf(name, sizeof(name), "%s/%s_%04d.csv", out.c_str(), kinds[k], files.start_image);
    if (rihvr_write_centroids(name, objs.data(), n, k == 1, k == 2) != RIHVR_OK)
      return fail_msg(rihvr_last_error());
  }
  return true;
}

int run(int argc, char** argv) {
  std::string param_file;
  bool subfolder = false, segment = false;
  int c;
  while ((c = getopt(argc, argv, "F:S:G:")) != -1) {
    switch (c) {
      case 'F': param_file = optarg; break;
      case 'S': subfolder = std::atoi(optarg) != 0; break;
      case 'G': segment = std::atoi(optarg) != 0; break;
      default: std::printf("Unknown input argument\n"); return -1;
    }
  }
  if (param_file.empty()) {
    std::printf("User must give input parameter file using -F flag\n");
    return -1;
  }
  rihvr_params p;
  rihvr_params_default(&p);
  rihvr_file_params files;
  int rc = rihvr_read_param_file(param_file.c_str(), &p, &files);
  if (rc != RIHVR_OK) return fail_msg(std::string("reading ") + param_file + ": " + rihvr_status_string(rc)), -1;
  char read_name[4096];
  std::snprintf(read_name, sizeof(read_name), files.image_filename, files.start_image);
  rihvr_io::Image holo, bg;
  std::string err;
  if (!rihvr_io::read_image(read_name, holo, err)) return fail_msg(err), -1;
  if (files.remove_background && !rihvr_io::read_image(files.background_filename, bg, err)) return fail_msg(err), -1;
  // the raw frame goes to the GPU as stored and is preprocessed there
  // (rihvr_set_hologram_frame); the size follows from the crop and padding
  rihvr_io::Preprocess pp;
  pp.roi_x = files.roi_x;
  pp.roi_y = files.roi_y;
  pp.roi_size = files.roi_size;
  pp.roi_rect_x = files.roi_rect_x;
  pp.roi_rect_y = files.roi_rect_y;
  pp.roi_rect_w = files.roi_rect_w;
  pp.roi_rect_h = files.roi_rect_h;
  if (files.remove_background && (bg.width != holo.width || bg.height != holo.height))
    return fail_msg("background must match the hologram size"), -1;
  const rihvr_io::CropRect cr = rihvr_io::crop_rect(pp, holo.width, holo.height);
  const int W = cr.w + 2 * p.zero_padding, H = cr.h + 2 * p.zero_padding;
  const std::string out = files.output_path;

  rihvr_ctx* ctx = nullptr;
  rc = rihvr_create(&p, W, H, &ctx);
  if (rc != RIHVR_OK) return fail_msg(std::string("rihvr_create: ") + rihvr_last_error()), -1;
  auto done = [&](int code) {
    rihvr_destroy(ctx);
    return code;
  };
  {
    // 8- and 16-bit frames travel as such; anything else as float samples
    const int bits = (holo.bits == 8 || holo.bits == 16) && (!files.remove_background || bg.bits == holo.bits)
                         ? holo.bits : 32;
    std::vector<unsigned char> fb, bb;
    auto pack = [&](const rihvr_io::Image& im, std::vector<unsigned char>& dst) {
      const size_t n = im.pixels.size();
      dst.resize(n * (bits / 8));
      for (size_t i = 0; i < n; ++i) {
        if (bits == 8) dst[i] = (unsigned char)im.pixels[i];
        else if (bits == 16) reinterpret_cast<unsigned short*>(dst.data())[i] = (unsigned short)im.pixels[i];
        else reinterpret_cast<float*>(dst.data())[i] = im.pixels[i];
      }
    };
    pack(holo, fb);
    if (files.remove_background) pack(bg, bb);
    if (rihvr_set_hologram_frame(ctx, fb.data(), bits, holo.width, holo.height,
                                 files.remove_background ? bb.data() : nullptr, &files, 0) != RIHVR_OK)
      return fail_msg(rihvr_last_error()), done(-1);
  }
  std::vector<float> b((size_t)W * H);
  if (rihvr_get_hologram(ctx, b.data(), 0) != RIHVR_OK) return fail_msg(rihvr_last_error()), done(-1);
  if (!write_minmax(out + "/enh.tif", b, W, H)) return done(-1);
  // calcInitialObjectiveFunction's images (sparse_compressive_holo.cu:2901-2966), limits +-0.25
  std::vector<float> est(b.size()), res(b.size());
  if (rihvr_initial_estimate(ctx, est.data(), 0) != RIHVR_OK) return fail_msg(rihvr_last_error()), done(-1);
  for (size_t i = 0; i < b.size(); ++i) res[i] = est[i] - b[i];
  write_scaled(out + "/initial_residual.tif", res, W, H, -0.25, 0.25);
  write_scaled(out + "/estimate_initial.tif", est, W, H, -0.25, 0.25);
  write_scaled(out + "/initial_measured.tif", b, W, H, -0.25, 0.25);

  FILE* metrics = std::fopen((out + "/all_metrics.csv").c_str(), "a");
  if (!metrics) return fail_msg("Unable to open file: " + out + "/all_metrics.csv"), done(-1);
  std::fprintf(metrics, "it, f, sparsity, stepsize, total_backtracks\n");
  // Without per-step outputs the iterations run in one call, which keeps them
  // on the device (one host synchronisation per 256 iterations) and reads the
  // log once at the end.  With output_steps the reference writes the sparsity
  // of every iterate (:586-589), which needs the volume after each iteration.
  const int n_iter = p.num_inverse_iterations;
  std::vector<rihvr_iter_record> recs((size_t)std::max(n_iter, 1));
  std::vector<double> sparsity((size_t)std::max(n_iter, 1), 0.0);
  for (int it = 0; it < n_iter;) {
    const int step = files.output_steps ? 1 : n_iter;
    if (rihvr_iterate(ctx, step) != RIHVR_OK) {
      std::fclose(metrics);
      return fail_msg(rihvr_last_error()), done(-1);
    }
    it += step;
    if (files.output_steps) rihvr_sparsity(ctx, &sparsity[(size_t)it - 1]);
  }
  int n_rec = 0;
  if (rihvr_get_iterations(ctx, recs.data(), n_iter, &n_rec) != RIHVR_OK) {
    std::fclose(metrics);
    return fail_msg(rihvr_last_error()), done(-1);
  }
  int total_bt = 0;
  for (int it = 0; it < n_rec; ++it) {
    const rihvr_iter_record& r = recs[(size_t)it];
    total_bt += r.backtracks;
    std::printf("FASTA iteration %d of %d: new f = %e, backtracks %d, stepsize %g%s\n", it + 1, n_iter, r.f_x,
                total_bt, r.t, r.restarted ? ", restarted" : "");
    if (files.output_steps)
      std::fprintf(metrics, "%d, %f, %f, %f, %d\n", it, r.f_x, sparsity[(size_t)it], r.t, total_bt);
  }
  std::fclose(metrics);
  const auto mm = std::minmax_element(b.begin(), b.end());
  rihvr_get_estimate(ctx, est.data(), 0);
  rihvr_get_residual(ctx, res.data(), 0);
  write_scaled(out + "/estimate_final.tif", est, W, H, *mm.first, *mm.second);
  write_scaled(out + "/residual_final.tif", res, W, H, *mm.first, *mm.second);

  Planes pl{ctx, W, H, p.num_planes, {}};
  std::string planes_prefix;
  if (files.output_planes) {
    planes_prefix = out + "/inverse";
    if (subfolder) {
      char sub[4096];
      std::snprintf(sub, sizeof(sub), "%s/%04d/", out.c_str(), files.start_image);
      mkdir(sub, 0755);
      planes_prefix = std::string(sub) + "inverse";
    }
  }
  if (!save_volume_outputs(pl, planes_prefix, out, "cmb", "inverse_voxels")) return done(-1);
  if (segment && !segment_and_save(ctx, files, out)) return done(-1);
  std::printf("Done.\n");
  return done(0);
}

}  // namespace

int main(int argc, char** argv) { return run(argc, argv); }
