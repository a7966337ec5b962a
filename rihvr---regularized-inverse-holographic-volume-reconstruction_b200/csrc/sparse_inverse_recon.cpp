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

bool magnitude_range(Planes& pl, double& lo, double& hi) {
  lo = hi = 0;
  for (int z = 0; z < pl.Nz; ++z) {
    const auto* p = pl.get(z);
    if (!p) return fail_msg(rihvr_last_error());
    double a = 1e300, b = -1e300;
    for (size_t i = 0; i < (size_t)pl.W * pl.H; ++i) {
      const double m = std::abs(p[i]);
      a = std::min(a, m);
      b = std::max(b, m);
    }
    if (z == 0) { lo = a; hi = b; }
    lo = std::min(lo, a);
    hi = std::max(hi, b);
  }
  return true;
}

// SparseCompressiveHolo::savePlanes (sparse_compressive_holo.cu:1039-1194)
bool save_planes(Planes& pl, const std::string& prefix) {
  double gmin, gmax;
  if (!magnitude_range(pl, gmin, gmax)) return false;
  const size_t n = (size_t)pl.W * pl.H;
  std::vector<uint8_t> px(n);
  std::string err;
  const double rmax = std::sqrt(gmax) / 10.0, rmin = -rmax;
  char name[4096];
  for (int z = 0; z < pl.Nz; ++z) {
    const auto* p = pl.get(z);
    if (!p) return fail_msg(rihvr_last_error());
    for (size_t i = 0; i < n; ++i) px[i] = to_u8((std::abs(p[i]) - gmin) / (gmax - gmin) * 255.0);
    std::snprintf(name, sizeof(name), "%s_%04d.tif", prefix.c_str(), z);
    if (!rihvr_io::write_tiff8(name, px.data(), pl.W, pl.H, err)) return fail_msg(err);
    for (size_t i = 0; i < n; ++i) {
      double ph = std::atan2((double)p[i].imag(), (double)p[i].real());  // cv::phase: [0, 2 pi)
      if (ph < 0) ph += 2.0 * M_PI;
      px[i] = to_u8(ph / (2.0 * M_PI) * 255.0);
    }
    std::snprintf(name, sizeof(name), "%s_phase_%04d.tif", prefix.c_str(), z);
    if (!rihvr_io::write_tiff8(name, px.data(), pl.W, pl.H, err)) return fail_msg(err);
    for (size_t i = 0; i < n; ++i) px[i] = to_u8((p[i].real() - rmin) / (rmax - rmin) * 255.0);
    std::snprintf(name, sizeof(name), "%s_real_%04d.tif", prefix.c_str(), z);
    if (!rihvr_io::write_tiff8(name, px.data(), pl.W, pl.H, err)) return fail_msg(err);
    for (size_t i = 0; i < n; ++i) px[i] = to_u8((p[i].imag() - rmin) / (rmax - rmin) * 255.0);
    std::snprintf(name, sizeof(name), "%s_imag_%04d.tif", prefix.c_str(), z);
    if (!rihvr_io::write_tiff8(name, px.data(), pl.W, pl.H, err)) return fail_msg(err);
  }
  return true;
}

// SparseVolume::saveProjections, MAX_CMB (sparse_volume.cu:684-813).  The
// reference starts the XY projection from zeros and folds in planes z > 0 only.
bool save_projections(Planes& pl, const std::string& output_path, const std::string& prefix) {
  double gmin, gmax;
  if (!magnitude_range(pl, gmin, gmax)) return false;
  const int W = pl.W, H = pl.H, Z = pl.Nz;
  std::vector<float> xy((size_t)W * H, 0.f), xz((size_t)Z * W, 0.f), yz((size_t)H * Z, 0.f);
  for (int z = 0; z < Z; ++z) {
    const auto* p = pl.get(z);
    if (!p) return fail_msg(rihvr_last_error());
    std::vector<float> colmax(W, -1e30f);
    for (int y = 0; y < H; ++y) {
      float rowmax = -1e30f;
      for (int x = 0; x < W; ++x) {
        const float v = (float)((std::abs(p[(size_t)y * W + x]) - gmin) / (gmax - gmin));
        rowmax = std::max(rowmax, v);
        colmax[x] = std::max(colmax[x], v);
        if (z > 0) xy[(size_t)y * W + x] = std::max(xy[(size_t)y * W + x], v);
      }
      yz[(size_t)y * Z + z] = rowmax;
    }
    for (int x = 0; x < W; ++x) xz[(size_t)z * W + x] = colmax[x];
  }
  auto put = [&](const std::vector<float>& v, int w, int h, const std::string& tag) {
    std::vector<uint8_t> px(v.size());
    for (size_t i = 0; i < v.size(); ++i) px[i] = to_u8(v[i] * 255.0);
    std::string err;
    const std::string name = output_path + prefix + "_" + tag + ".tif";  // no separator, as the reference
    return rihvr_io::write_tiff8(name, px.data(), w, h, err) || fail_msg(err);
  };
  return put(xy, W, H, "xy") && put(xz, W, Z, "xz") && put(yz, Z, H, "yz");
}

// SparseVolume::saveData (sparse_volume.cu:518-560): non-zero voxels with
// their intensity, plane by plane (raster order within a plane).
bool save_sparse(Planes& pl, const std::string& output_path, const std::string& prefix) {
  const std::string name = output_path + "/" + prefix + ".csv";
  FILE* f = std::fopen(name.c_str(), "w");
  if (!f) return fail_msg("Unable to open file: " + name);
  std::fprintf(f, "x, y, z, value\n");
  for (int z = 0; z < pl.Nz; ++z) {
    const auto* p = pl.get(z);
    if (!p) {
      std::fclose(f);
      return fail_msg(rihvr_last_error());
    }
    for (int y = 0; y < pl.H; ++y)
      for (int x = 0; x < pl.W; ++x) {
        const std::complex<float> v = p[(size_t)y * pl.W + x];
        if (v.real() == 0.f && v.imag() == 0.f) continue;
        const float intensity = v.real() * v.real() + v.imag() * v.imag();
        std::fprintf(f, "%d, %d, %d, %e\n", x, y, z, intensity);
      }
  }
  std::fclose(f);
  return true;
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
  rihvr_io::Preprocess pp;
  pp.remove_background = files.remove_background;
  pp.roi_x = files.roi_x;
  pp.roi_y = files.roi_y;
  pp.roi_size = files.roi_size;
  pp.roi_rect_x = files.roi_rect_x;
  pp.roi_rect_y = files.roi_rect_y;
  pp.roi_rect_w = files.roi_rect_w;
  pp.roi_rect_h = files.roi_rect_h;
  pp.zero_padding = p.zero_padding;
  std::vector<float> b;
  int W, H;
  if (!rihvr_io::preprocess(holo, files.remove_background ? &bg : nullptr, pp, b, W, H, err)) return fail_msg(err), -1;
  const std::string out = files.output_path;
  if (!write_minmax(out + "/enh.tif", b, W, H)) return -1;

  rihvr_ctx* ctx = nullptr;
  rc = rihvr_create(&p, W, H, &ctx);
  if (rc != RIHVR_OK) return fail_msg(std::string("rihvr_create: ") + rihvr_last_error()), -1;
  auto done = [&](int code) {
    rihvr_destroy(ctx);
    return code;
  };
  if (rihvr_set_hologram(ctx, b.data(), 0) != RIHVR_OK) return fail_msg(rihvr_last_error()), done(-1);
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
  int total_bt = 0;
  for (int it = 0; it < p.num_inverse_iterations; ++it) {
    if (rihvr_iterate(ctx, 1) != RIHVR_OK) {
      std::fclose(metrics);
      return fail_msg(rihvr_last_error()), done(-1);
    }
    std::vector<rihvr_iter_record> recs(it + 1);
    int n = 0;
    rihvr_get_iterations(ctx, recs.data(), it + 1, &n);
    const rihvr_iter_record& r = recs[it];
    total_bt += r.backtracks;
    double sparsity = 0;
    if (files.output_steps) rihvr_sparsity(ctx, &sparsity);
    std::printf("FASTA iteration %d of %d: new f = %e, backtracks %d, stepsize %g%s\n", it + 1,
                p.num_inverse_iterations, r.f_x, total_bt, r.t, r.restarted ? ", restarted" : "");
    if (files.output_steps)
      std::fprintf(metrics, "%d, %f, %f, %f, %d\n", it, r.f_x, sparsity, r.t, total_bt);
  }
  std::fclose(metrics);
  const auto mm = std::minmax_element(b.begin(), b.end());
  rihvr_get_estimate(ctx, est.data(), 0);
  rihvr_get_residual(ctx, res.data(), 0);
  write_scaled(out + "/estimate_final.tif", est, W, H, *mm.first, *mm.second);
  write_scaled(out + "/residual_final.tif", res, W, H, *mm.first, *mm.second);

  Planes pl{ctx, W, H, p.num_planes, {}};
  if (files.output_planes) {
    std::string prefix = out + "/inverse";
    if (subfolder) {
      char sub[4096];
      std::snprintf(sub, sizeof(sub), "%s/%04d/", out.c_str(), files.start_image);
      mkdir(sub, 0755);
      prefix = std::string(sub) + "inverse";
    }
    if (!save_planes(pl, prefix)) return done(-1);
  }
  if (!save_projections(pl, out, "cmb")) return done(-1);
  if (!save_sparse(pl, out, "inverse_voxels")) return done(-1);
  if (segment && !segment_and_save(ctx, files, out)) return done(-1);
  std::printf("Done.\n");
  return done(0);
}

}  // namespace

int main(int argc, char** argv) { return run(argc, argv); }
