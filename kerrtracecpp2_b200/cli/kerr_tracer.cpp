// kerr_tracer -- command-line front end of the B200 renderer.
//
// Accepts the reference renderer's flags (main.cpp:2548-2678) for the
// single-frame and two-phase modes and drives the C ABI:
//   single frame : trace + colour on the GPU, PNG out (render_image)
//   --geo-only   : trace, write the .kgeo cache (trace_geodesics + save_kgeo)
//   --color-only : read a .kgeo file, colour it, PNG out (colorize_buffer)
// Flag meaning and defaults follow the reference: a=0.998, theta=80, phi=0,
// r_obs=40, fov=30, disk_out=12, 1920x1080, KS chart, RK4 doubling, tol
// 1e-7, step_init 1, max_steps 500000; --ks/--bl/--chart, --dopri5,
// --bundles, --gpu-fp64 (always true here), --solver-mode standard.
// Backgrounds: the reference's default photograph is not in its tree, so the
// default is the seed-0 procedural star field; --bg accepts binary PPM (P6)
// or procedural:SEED.  --print-config prints the parsed frame as JSON and
// exits without tracing.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "../../include/kerrtrace.h"

namespace {

// ---------------------------------------------------------------- PNG out
// Minimal PNG encoder: RGB8, zlib stream of stored (uncompressed) deflate
// blocks, CRC-32 and Adler-32 computed here.
uint32_t crc_table[256];
void crc_init() {
  for (uint32_t n = 0; n < 256; ++n) {
    uint32_t c = n;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
    crc_table[n] = c;
  }
}
uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xffffffffu) {
  for (size_t i = 0; i < n; ++i) c = crc_table[(c ^ p[i]) & 0xff] ^ (c >> 8);
  return c;
}
void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back(x >> 24);
  v.push_back(x >> 16);
  v.push_back(x >> 8);
  v.push_back(x);
}
void chunk(FILE* f, const char* type, const std::vector<uint8_t>& data) {
  std::vector<uint8_t> buf;
  put32(buf, (uint32_t)data.size());
  buf.insert(buf.end(), type, type + 4);
  buf.insert(buf.end(), data.begin(), data.end());
  const uint32_t c = crc32(buf.data() + 4, buf.size() - 4) ^ 0xffffffffu;
  put32(buf, c);
  fwrite(buf.data(), 1, buf.size(), f);
}
bool write_png(const char* path, const uint8_t* rgb, int W, int H) {
  crc_init();
  FILE* f = fopen(path, "wb");
  if (!f) return false;
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  fwrite(sig, 1, 8, f);
  std::vector<uint8_t> ihdr;
  put32(ihdr, W);
  put32(ihdr, H);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
  chunk(f, "IHDR", ihdr);
  std::vector<uint8_t> raw;
  raw.reserve((size_t)H * (3 * (size_t)W + 1));
  for (int y = 0; y < H; ++y) {
    raw.push_back(0);  // filter: none
    raw.insert(raw.end(), rgb + (size_t)y * W * 3, rgb + (size_t)(y + 1) * W * 3);
  }
  std::vector<uint8_t> z = {0x78, 0x01};
  uint32_t a = 1, b = 0;
  for (uint8_t c : raw) {
    a = (a + c) % 65521;
    b = (b + a) % 65521;
  }
  for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
    const size_t len = std::min<size_t>(65535, raw.size() - off);
    z.push_back(off + len >= raw.size() ? 1 : 0);
    z.push_back(len & 0xff);
    z.push_back(len >> 8);
    z.push_back(~len & 0xff);
    z.push_back((~len >> 8) & 0xff);
    z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
    if (raw.empty()) break;
  }
  put32(z, (b << 16) | a);
  chunk(f, "IDAT", z);
  chunk(f, "IEND", {});
  return fclose(f) == 0;
}

// ---------------------------------------------------------- backgrounds
bool read_ppm(const char* path, std::vector<uint8_t>& px, int& w, int& h) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  char magic[3] = {0};
  int maxv = 0;
  bool ok = fscanf(f, "%2s %d %d %d", magic, &w, &h, &maxv) == 4 && strcmp(magic, "P6") == 0 &&
            maxv == 255 && w > 0 && h > 0;
  if (ok) {
    fgetc(f);
    px.resize((size_t)w * h * 3);
    ok = fread(px.data(), 1, px.size(), f) == px.size();
  }
  fclose(f);
  return ok;
}

bool load_background(const std::string& spec, std::vector<uint8_t>& px, int& w, int& h) {
  if (spec.rfind("procedural:", 0) == 0 || spec.empty()) {
    const uint64_t seed = spec.empty() ? 0 : strtoull(spec.c_str() + 11, nullptr, 10);
    w = 2048;
    h = 1024;
    px.resize((size_t)w * h * 3);
    return kt_starfield(seed, w, h, px.data()) == KT_OK;
  }
  return read_ppm(spec.c_str(), px, w, h);
}

double now_s() {
  using C = std::chrono::steady_clock;
  return std::chrono::duration<double>(C::now().time_since_epoch()).count();
}

std::string timestamp() {
  std::time_t t = std::time(nullptr);
  char ts[32];
  std::strftime(ts, sizeof ts, "%Y%m%d-%H%M%S", std::localtime(&t));
  return ts;
}

int die(const char* what, kt_context* ctx, kt_status st) {
  fprintf(stderr, "Error: %s: %s (%s)\n", what, ctx ? kt_last_error(ctx) : "",
          kt_status_string(st));
  if (ctx) kt_destroy(ctx);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  kt_frame_desc d;
  kt_frame_desc_defaults(&d);
  kt_color_params cp;
  kt_color_params_defaults(&cp);
  bool preview = false, hd = false, r720 = false, r2k = false, r4k = false;
  int custom_w = 0, custom_h = 0;
  bool geo_only = false, color_only = false, print_config = false;
  std::string geo_file, bg_spec, out_path, out_dir = "out";
  double arg_r_obs = -1.0;
  int camera_spp = 1;
  bool debug_elliptic = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a(argv[i]);
    auto next = [&](void) -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "Error: %s needs a value\n", a.c_str());
        exit(2);
      }
      return argv[++i];
    };
    if (a == "--bundles") d.bundles = 1;
    // extension: trace bundle rays creeping onto the horizon to the
    // reference's reject or step cap (its step counts; same image either way)
    else if (a == "--bundle-full-creep") d.flags |= KT_FLAG_BUNDLE_FULL_CREEP;
    else if (a == "--dopri5") d.integrator = KT_DOPRI5;
    else if (a == "--max-steps") d.max_steps = std::max(1, atoi(next()));
    else if (a == "--step-init" || a == "--step-size") d.step_init = atof(next());
    else if (a == "--integrator-tol" || a == "--tol") d.tol = atof(next());
    else if (a == "--camera-spp" || a == "--spp") camera_spp = std::max(1, atoi(next()));
    else if (a == "--semi-analytic" || a == "--elliptic") d.solver_mode = KT_SOLVER_SEMI_ANALYTIC;
    else if (a == "--elliptic-closed") d.solver_mode = KT_SOLVER_ELLIPTIC_CLOSED;
    else if (a == "--solver-mode") {
      const std::string s = next();
      if (s == "standard") d.solver_mode = KT_SOLVER_STANDARD;
      else if (s == "semi" || s == "semi-analytic" || s == "semi_analytic") d.solver_mode = KT_SOLVER_SEMI_ANALYTIC;
      else if (s == "elliptic" || s == "elliptic-closed" || s == "elliptic_closed") d.solver_mode = KT_SOLVER_ELLIPTIC_CLOSED;
    } else if (a == "--gpu-fp64" || a == "--gpu-fp64-on" || a == "--metal-fp64" || a == "--cuda-fp64" ||
               a == "--no-gpu-fp64" || a == "--no-cuda-fp64") {
      // this backend always traces in FP64
    } else if (a == "--bl") d.chart = KT_CHART_BL;
    else if (a == "--ks") d.chart = KT_CHART_KS;
    else if (a == "--chart") {
      const std::string c = next();
      if (c == "bl" || c == "BL") d.chart = KT_CHART_BL;
      else if (c == "ks" || c == "KS") d.chart = KT_CHART_KS;
    } else if (a == "--intersection-hermite" || a == "--hermite-intersection") {
    } else if (a == "--intersection-linear" || a == "--linear-intersection") {
      fprintf(stderr, "Info: the CPU path always locates events by Hermite interpolation; "
                      "--intersection-linear only affected the Metal backend.\n");
    } else if (a == "--intersection") next();
    else if (a == "--preview") preview = true;
    else if (a == "--hd") hd = true;
    else if (a == "--720p") r720 = true;
    else if (a == "--2k") r2k = true;
    else if (a == "--4k") r4k = true;
    else if (a == "--custom-res") {
      custom_w = atoi(next());
      custom_h = atoi(next());
    } else if (a == "--bg") bg_spec = next();
    else if (a == "--a") d.a = atof(next());
    else if (a == "--disk-out") d.disk_out = atof(next());
    else if (a == "--theta") d.theta_deg = atof(next());
    else if (a == "--phi") d.phi_deg = atof(next());
    else if (a == "--r-obs") arg_r_obs = atof(next());
    else if (a == "--charge") d.Q = atof(next());
    else if (a == "--lambda") d.Lambda = atof(next());
    else if (a == "--fov") d.fov_deg = atof(next());
    else if (a == "--exposure") cp.exposure = atof(next());
    else if (a == "--gamma") cp.gamma = atof(next());
    else if (a == "--temp-scale") cp.temp_scale = atof(next());
    else if (a == "--disk-interstellar") cp.palette = 1;
    else if (a == "--disk-blackbody") cp.palette = 0;
    else if (a == "--debug-elliptic") debug_elliptic = true;
    else if (a == "--anti-fireflies" || a == "--anti_fireflies" || a == "--no-anti-fireflies" ||
             a == "--no-anti_fireflies" || a == "--elliptic-fallback-black" ||
             a == "--elliptic-strict-black") {
      // Metal-backend options: the reference's CPU path ignores them (main.cpp:2327-2328)
    } else if (a == "--metal-kernel") next();
    else if (a == "--disk-rings") cp.disk_rings = atoi(next());
    else if (a == "--disk-sectors") cp.disk_sectors = atoi(next());
    else if (a == "--disk-sigma") cp.disk_sigma = atof(next());
    else if (a == "--disk-hue-offset") cp.disk_hue_offset = atof(next());
    else if (a == "--geo-only") geo_only = true;
    else if (a == "--geo-file") geo_file = next();
    else if (a == "--color-only") {
      color_only = true;
      geo_file = next();
    } else if (a == "--output") out_path = next();
    else if (a == "--out-dir") out_dir = next();
    else if (a == "--print-config") print_config = true;
    else if (a == "--anim" || a == "--wormhole") {
      fprintf(stderr, "Error: %s is not part of this backend (single-frame geodesic path only)\n", a.c_str());
      return 2;
    } else {
      fprintf(stderr, "Warning: ignoring unknown argument '%s'\n", a.c_str());
    }
  }
  // main.cpp:2683-2716
  d.max_steps = std::max(1, (int)d.max_steps);
  d.step_init = std::max(1e-10, d.step_init);
  d.tol = std::max(1e-10, d.tol);
  d.width = custom_w ? custom_w : r4k ? 3840 : r2k ? 2560 : r720 ? 1280 : hd ? 854 : preview ? 480 : 1920;
  d.height = custom_h ? custom_h : r4k ? 2160 : r2k ? 1440 : r720 ? 720 : hd ? 480 : preview ? 270 : 1080;
  d.r_obs = (arg_r_obs > 0) ? arg_r_obs : 40.0;

  if (print_config) {
    printf("{\"M\": %.17g, \"a\": %.17g, \"Q\": %.17g, \"Lambda\": %.17g, \"theta_deg\": %.17g, "
           "\"phi_deg\": %.17g, \"r_obs\": %.17g, \"disk_out\": %.17g, \"fov_deg\": %.17g, "
           "\"width\": %d, \"height\": %d, \"chart\": %d, \"integrator\": %d, \"bundles\": %d, "
           "\"solver_mode\": %d, \"max_steps\": %d, \"step_init\": %.17g, \"tol\": %.17g, "
           "\"camera_spp\": %d, \"exposure\": %.17g, \"gamma\": %.17g, \"temp_scale\": %.17g, "
           "\"palette\": %d, \"disk_rings\": %d, \"disk_sectors\": %d, \"disk_sigma\": %.17g, "
           "\"disk_hue_offset\": %.17g}\n",
           d.M, d.a, d.Q, d.Lambda, d.theta_deg, d.phi_deg, d.r_obs, d.disk_out, d.fov_deg, d.width,
           d.height, d.chart, d.integrator, d.bundles, d.solver_mode, d.max_steps, d.step_init, d.tol,
           camera_spp, cp.exposure, cp.gamma, cp.temp_scale, cp.palette, cp.disk_rings,
           cp.disk_sectors, cp.disk_sigma, cp.disk_hue_offset);
    return 0;
  }
  if (camera_spp > KT_MAX_CAMERA_SPP) {
    fprintf(stderr, "Error: --camera-spp above %d is not supported\n", KT_MAX_CAMERA_SPP);
    return 2;
  }

  std::vector<uint8_t> bg;
  int bw = 0, bh = 0;
  if (!load_background(bg_spec, bg, bw, bh)) {
    fprintf(stderr, "Warning: cannot load background '%s' (binary PPM or procedural:SEED)\n",
            bg_spec.c_str());
    bg.clear();
  }
  kt_context* ctx = nullptr;
  kt_status st = kt_create(&ctx, 0);
  if (st != KT_OK) return die("kt_create", nullptr, st);
  system(("mkdir -p \"" + out_dir + "\"").c_str());

  if (color_only) {
    int32_t W = 0, H = 0;
    double meta[10];
    st = kt_kgeo_read_header(geo_file.c_str(), &W, &H, meta);
    if (st != KT_OK) return die("cannot read .kgeo header", ctx, st);
    const size_t n = (size_t)W * H;
    std::vector<uint8_t> oc(n);
    std::vector<double> f6(6 * n);
    kt_geo_soa g = {oc.data(), &f6[0], &f6[n], &f6[2 * n], &f6[3 * n], &f6[4 * n], &f6[5 * n],
                    nullptr, nullptr, nullptr};
    st = kt_kgeo_read(geo_file.c_str(), &g, (int64_t)n);
    if (st != KT_OK) return die("cannot read .kgeo", ctx, st);
    printf("Loaded: %s  %dx%d  a=%g  r_isco=%g\n", geo_file.c_str(), W, H, meta[1], meta[4]);
    std::vector<uint8_t> rgb(3 * n);
    st = kt_colorize_host(ctx, &g, W, H, meta[0], meta[4], meta[5], meta[6], &cp,
                          bg.empty() ? nullptr : bg.data(), bw, bh, rgb.data());
    if (st != KT_OK) return die("colorize", ctx, st);
    std::string base = geo_file;
    if (base.size() > 5 && base.substr(base.size() - 5) == ".kgeo") base = base.substr(0, base.size() - 5);
    const std::string png = out_path.empty() ? base + "_recolor_" + timestamp() + ".png" : out_path;
    if (!write_png(png.c_str(), rgb.data(), W, H)) return die("cannot write PNG", ctx, KT_ERR_IO);
    printf("Saved: %s\n", png.c_str());
    kt_destroy(ctx);
    return 0;
  }

  kt_frame_derived dv;
  st = kt_frame_derive(&d, &dv);
  if (st != KT_OK) return die("invalid frame", ctx, st);
  printf("KNdS  M=%g a=%g Q=%g Lambda=%g\n  r+=%.10g  r_ISCO=%.10g\n", d.M, d.a, d.Q, d.Lambda,
         dv.r_horizon, dv.r_isco);
  static const char* const kSolverName[] = {"standard", "semi-analytic", "elliptic-closed"};
  if (dv.solver != d.solver_mode)  // select_solver_mode's fallback (main.cpp:2051-2060)
    fprintf(stderr, "Info: requested solver '%s' not available here; using standard integrator.\n",
            kSolverName[d.solver_mode]);
  printf("Mode: %s  chart=%s  %s  %s  backend=gpu-b200  tol=%g  max-steps=%d  %dx%d\n",
         d.bundles ? "ray bundles" : "single ray", dv.chart == KT_CHART_KS ? "KS" : "BL",
         dv.solver == KT_SOLVER_SEMI_ANALYTIC ? "RK4-doubling"
         : dv.integrator == KT_DOPRI5         ? "DOPRI5"
                                              : "RK4-doubling",
         kSolverName[dv.solver], d.tol, d.max_steps, d.width, d.height);
  const size_t n = (size_t)d.width * d.height;
  const std::string spp_tag = camera_spp > 1 ? "_spp" + std::to_string(camera_spp) : "";
  const std::string tag = std::string(d.bundles ? "bundles" : "trace") + "_" +
                          std::to_string(d.width) + "x" + std::to_string(d.height) + "_" +
                          (dv.chart == KT_CHART_KS ? "ks" : "bl") + "_gpu-b200" + spp_tag + "_" +
                          timestamp();
  const double t0 = now_s();
  // main.cpp:2897-2945: --geo-only traces and saves the .kgeo (camera_spp
  // plays no part); a full render with --geo-file also saves the frame's
  // .kgeo beside the PNG, except with camera_spp > 1 (main.cpp:2232-2236).
  const bool save_geo = geo_only || (!geo_file.empty() && camera_spp <= 1);
  if (!geo_only && !geo_file.empty() && camera_spp > 1)
    fprintf(stderr, "Info: camera-spp>1 uses jittered multi-pass sampling and disables .kgeo export "
                    "for this frame.\n");
  std::vector<uint8_t> oc, rgb;
  std::vector<double> f6;
  kt_geo_soa g = {};
  if (save_geo) {
    oc.resize(n);
    f6.resize(6 * n);
    g = {oc.data(), &f6[0], &f6[n], &f6[2 * n], &f6[3 * n], &f6[4 * n], &f6[5 * n], nullptr, nullptr,
         nullptr};
    st = kt_trace_host(ctx, &d, &g);
    if (st != KT_OK) return die("trace", ctx, st);
  }
  if (!geo_only) {
    rgb.resize(3 * n);
    if (debug_elliptic) {
      // colorize_buffer's debug branch (main.cpp:1828-1843): the colour of
      // the elliptic-closed solver's fallback reason
      static const uint8_t kTag[KT_ELLIPTIC_REASONS][3] = {
          {0, 220, 0}, {255, 255, 255}, {0, 220, 220}, {220, 0, 0}, {220, 220, 0}, {60, 60, 220}};
      std::vector<uint8_t> why(n);
      if (camera_spp > 1)
        fprintf(stderr, "Info: --debug-elliptic colours one pass (camera-spp ignored).\n");
      st = kt_elliptic_reasons_host(ctx, &d, why.data());
      for (size_t i = 0; st == KT_OK && i < n; ++i)
        for (int c = 0; c < 3; ++c) rgb[3 * i + c] = why[i] < KT_ELLIPTIC_REASONS ? kTag[why[i]][c] : (c == 1 ? 0 : 128);
    } else if (save_geo)
      st = kt_colorize_host(ctx, &g, d.width, d.height, d.M, dv.r_isco, dv.r_disk_in, dv.r_disk_out,
                            &cp, bg.empty() ? nullptr : bg.data(), bw, bh, rgb.data());
    else
      st = kt_render_spp_host(ctx, &d, &cp, camera_spp, bg.empty() ? nullptr : bg.data(), bw, bh,
                              rgb.data());
    if (st != KT_OK) return die("render", ctx, st);
  }
  const double el = now_s() - t0;
  printf("%s: %gs  (%.1f kpix/s)\n", geo_only ? "Trace" : "Time", el, n / el / 1e3);
  if (!geo_only) {
    const std::string png = out_path.empty() ? out_dir + "/" + tag + ".png" : out_path;
    if (!write_png(png.c_str(), rgb.data(), d.width, d.height)) return die("cannot write PNG", ctx, KT_ERR_IO);
    printf("Saved: %s\n", png.c_str());
  }
  if (save_geo) {
    const std::string path = geo_file.empty() ? out_dir + "/" + tag + ".kgeo" : geo_file;
    st = kt_kgeo_write(path.c_str(), &d, &g);
    if (st != KT_OK) return die("cannot write .kgeo", ctx, st);
    printf("Geo saved: %s\n", path.c_str());
  }
  kt_destroy(ctx);
  return 0;
}
