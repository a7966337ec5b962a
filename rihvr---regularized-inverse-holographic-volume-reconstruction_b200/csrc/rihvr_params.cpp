// Parameter defaults and the .param text format of RIHVR
// (HoloUi::HoloUi, src/core/holo_ui.cpp:10-62; HoloUi::readFile, :171-486;
// codes from src/core/holo_ui.h:22-78).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/rihvr.h"

namespace {
thread_local std::string g_param_error;
}

extern "C" {

int rihvr_params_default(rihvr_params* p) {
  if (!p) return RIHVR_ERR_INVALID_ARGUMENT;
  std::memset(p, 0, sizeof(*p));
  p->start_plane = 0.f;
  p->plane_stepsize = 1.0f;
  p->num_planes = 256;
  p->wavelength = 632.f;
  p->resolution = 1000.f;
  p->zero_padding = 256;
  p->num_inverse_iterations = 500;
  p->num_tv_iterations = 5;
  p->regularization_param = 0.01f;
  p->regularization_TV_param = 0.0f;
  p->mode = RIHVR_MODE_FASTA_FUSED_LASSO_2D;
  p->storage = RIHVR_STORE_F32;
  p->faithful = 1;
  p->max_backtracks = 2;
  p->initial_step = 0.0;
  p->record_objective = 1;
  p->autotune = 0;
  return RIHVR_OK;
}

int rihvr_plane_list(const rihvr_params* p, double* z) {
  if (!p || !z) return RIHVR_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < p->num_planes; ++i) {
    // float arithmetic, as holo_ui.cpp:481 (float z = start_plane + i * plane_stepsize)
    volatile float step = (float)i * p->plane_stepsize;
    volatile float zf = p->start_plane + step;
    z[i] = (double)zf;
  }
  return RIHVR_OK;
}

static void copy_str(char* dst, const char* src) { std::snprintf(dst, 4096, "%s", src); }

int rihvr_read_param_file(const char* path, rihvr_params* p, rihvr_file_params* f) {
  if (!path || !p) return RIHVR_ERR_INVALID_ARGUMENT;
  FILE* fid = std::fopen(path, "r");
  if (!fid) return RIHVR_ERR_BAD_FILENAME;
  rihvr_file_params local;
  if (!f) f = &local;
  std::memset(f, 0, sizeof(*f));
  f->roi_x = f->roi_y = f->roi_size = -1;  // whole image (HoloUi defaults, holo_ui.cpp:17-20)
  f->segment_min_area = 2;                  // segmentation defaults (holo_ui.cpp:44-46)
  f->segment_min_intensity = 1.0;
  f->segment_close_size = 3;
  f->background_start = f->background_end = -1;  // holo_ui.cpp:28-29
  bool set_full_filename = false;
  char buff[8192];
  char description[8192];
  char char_value[8192];
  int status = RIHVR_OK;
  while (std::fgets(buff, sizeof(buff), fid)) {
    if (buff[0] == '%' || buff[0] == '#') continue;
    int id = 0;
    float value = 0.f;
    char_value[0] = '\0';
    const int n1 = std::sscanf(buff, "%8191s %d %f", description, &id, &value);
    if (n1 < 2) continue;  // blank or malformed line
    std::sscanf(buff, "%8191s %d %8191[^\t\n]", description, &id, char_value);
    const bool is_true = std::strcmp(char_value, "true") == 0;
    const bool is_false = std::strcmp(char_value, "false") == 0;
    auto flag = [&](int* dst) { *dst = is_true ? 1 : is_false ? 0 : (value != 0.f); };
    switch (id) {
      case 1001: f->image_count = (int)value; break;
      case 1002: f->start_image = (int)value; break;
      case 1003: f->background_start = (int)value; break;
      case 1004: f->background_end = (int)value; break;
      case 2001: copy_str(f->image_filename, char_value); set_full_filename = true; break;
      case 2002: copy_str(f->image_path, char_value); break;
      case 2003: copy_str(f->image_formatted_name, char_value); break;
      case 2004: copy_str(f->output_path, char_value); break;
      case 2005: copy_str(f->background_filename, char_value); f->remove_background = 1; break;
      case 2006: break;  // executable path (GUI only)
      case 3001: p->start_plane = value; break;
      case 3002: p->plane_stepsize = value; break;
      case 3003: p->num_planes = (int)value; break;
      case 3004: p->wavelength = value; break;
      case 3005: p->resolution = value; break;
      case 3006: f->roi_x = (int)value; break;
      case 3007: f->roi_y = (int)value; break;
      case 3008: break;  // roi z (unused by the inverse path)
      case 3009: f->roi_size = (int)value; break;
      case 3010: p->zero_padding = (int)value; break;
      case 3011: f->roi_rect_x = (int)value; break;
      case 3012: f->roi_rect_y = (int)value; break;
      case 3013: f->roi_rect_w = (int)value; break;
      case 3014: f->roi_rect_h = (int)value; break;
      // 4001-5008: classic reconstruction and simulation settings
      case 4001: case 4002: case 5001: case 5002: case 5003: case 5004: case 5005:
      case 5006: case 5007: case 5008: break;
      case 5009: f->segment_min_area = (int)value; break;
      case 5010: f->segment_min_intensity = value; break;
      case 5011: f->segment_close_size = (int)value; break;
      case 6001: p->num_inverse_iterations = (int)value; break;
      case 6002: p->regularization_param = value; break;
      case 6003: break;  // max_svd (unused by the sparse solver)
      case 6004: p->regularization_TV_param = value; break;
      case 6005: p->num_tv_iterations = (int)value; break;
      case 7001: flag(&f->output_planes); break;
      case 7005: flag(&f->output_steps); break;
      case 7006: flag(&f->use_median_background); break;
      case 7002: case 7003: case 7004: break;  // other pipelines' switches
      default:
        // the reference prints and stops reading (:475-480); report it instead
        g_param_error = std::string("unknown or unsupported parameter line: ") + buff;
        status = RIHVR_ERR_INVALID_FILE;
        break;
    }
    if (status != RIHVR_OK) break;
  }
  std::fclose(fid);
  if (!set_full_filename) {
    std::string full = std::string(f->image_path) + f->image_formatted_name;
    copy_str(f->image_filename, full.c_str());
  }
  return status;
}

}  // extern "C"
