// sparse-segmentation: the reference's segmentation program
// (src/core/main_segmentation.cu:37-138): -F <file.param>.
//
// Reads the .param file and the hologram frame (its crop and zero padding
// give the volume's width and height, as Hologram::crop/zeroPad do there),
// loads <output_path>/inverse_voxels_XXXX.csv (SparseVolume::loadData,
// sparse_volume.cu:562-665: "x, y, z, value" with the voxel intensities),
// segments on the GPU through rihvr_segment_intensity and writes
// centroids_XXXX.csv, centroids_weighted_XXXX.csv and
// centroids_verbose_XXXX.csv (ObjectCloud::writeCentroids).
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rihvr.h"
#include "rihvr_image.h"

namespace {

int fail_msg(const std::string& m) {
  std::fprintf(stderr, "%s\n", m.c_str());
  return -1;
}

int run(int argc, char** argv) {
  std::string param_file;
  int c;
  while ((c = getopt(argc, argv, "F:")) != -1) {
    switch (c) {
      case 'F': param_file = optarg; break;
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
  if (rihvr_read_param_file(param_file.c_str(), &p, &files) != RIHVR_OK)
    return fail_msg(std::string("reading ") + param_file + ": " + rihvr_last_error());
  // volume size: the frame after crop and zero padding (main_segmentation.cu:91-98)
  char name[8192];
  std::snprintf(name, sizeof(name), files.image_filename, files.start_image);
  rihvr_io::Image holo;
  std::string err;
  if (!rihvr_io::read_image(name, holo, err)) return fail_msg(err);
  rihvr_io::Preprocess pp;
  pp.roi_x = files.roi_x;
  pp.roi_y = files.roi_y;
  pp.roi_size = files.roi_size;
  pp.roi_rect_x = files.roi_rect_x;
  pp.roi_rect_y = files.roi_rect_y;
  pp.roi_rect_w = files.roi_rect_w;
  pp.roi_rect_h = files.roi_rect_h;
  pp.zero_padding = p.zero_padding;
  std::vector<float> b;
  int W = 0, H = 0;
  if (!rihvr_io::preprocess(holo, nullptr, pp, b, W, H, err)) return fail_msg(err);
  const int Nz = p.num_planes;

  // SparseVolume::loadData: header, then "x, y, z, intensity" lines
  std::snprintf(name, sizeof(name), "%s/inverse_voxels_%04d.csv", files.output_path, files.start_image);
  FILE* f = std::fopen(name, "r");
  if (!f) return fail_msg(std::string("Unable to open file: ") + name);
  char header[64] = {0};
  if (!std::fgets(header, sizeof(header), f) || std::strncmp(header, "x, y, z, value", 14) != 0) {
    std::fclose(f);
    return fail_msg(std::string("File <") + name + "> is not correctly formatted");
  }
  std::vector<float> I((size_t)W * H * Nz, 0.f);
  int x, y, z;
  float v;
  long long count = 0;
  while (std::fscanf(f, "%d, %d, %d, %e\n", &x, &y, &z, &v) == 4) {
    if (x < 0 || x >= W || y < 0 || y >= H || z < 0 || z >= Nz) {
      std::fclose(f);
      std::fprintf(stderr, "Error: mismatch between loaded data and expected volume size\n");
      std::fprintf(stderr, "Expected width = %d, height = %d, depth = %d\n", W, H, Nz);
      std::fprintf(stderr, "Loaded voxel data at x = %d, y = %d, z = %d\n", x, y, z);
      return -1;
    }
    I[((size_t)z * H + y) * W + x] = v;
    ++count;
  }
  std::fclose(f);
  std::printf("loaded %lld voxels\n", count);

  rihvr_segment_params sp;
  rihvr_segment_params_default(&sp);
  sp.min_intensity = files.segment_min_intensity;
  sp.close_size = files.segment_close_size;
  sp.min_area = files.segment_min_area;
  std::vector<rihvr_object> objs(1 << 16);
  int n = 0;
  rihvr_segment_info info;
  int rc = rihvr_segment_intensity(I.data(), W, H, Nz, 0, &sp, objs.data(), (int)objs.size(), &n, &info);
  if (rc == RIHVR_ERR_INVALID_ARGUMENT && n > (int)objs.size()) {
    objs.resize(n);
    rc = rihvr_segment_intensity(I.data(), W, H, Nz, 0, &sp, objs.data(), (int)objs.size(), &n, &info);
  }
  if (rc != RIHVR_OK) return fail_msg(std::string("rihvr_segment_intensity: ") + rihvr_last_error());
  std::printf("max intensity = %f, thr = %f\n", info.max_intensity, info.threshold);
  std::printf("Number of particles: %lld\n", info.labelled_objects);
  std::printf("blobSizeFilter removed %lld objects\n", info.labelled_objects - n);
  const char* kinds[3] = {"centroids", "centroids_weighted", "centroids_verbose"};
  for (int k = 0; k < 3; ++k) {
    std::snprintf(name, sizeof(name), "%s/%s_%04d.csv", files.output_path, kinds[k], files.start_image);
    if (rihvr_write_centroids(name, objs.data(), n, k == 1, k == 2) != RIHVR_OK) return fail_msg(rihvr_last_error());
  }
  std::printf("Done.\n");
  return 0;
}

}  // namespace

int main(int argc, char** argv) { return run(argc, argv); }
