// kt_io.cpp -- host I/O of the C ABI: the .kgeo two-phase cache and the
// procedural background.
//
// .kgeo (save_kgeo / load_kgeo, main.cpp:96-137): "KGEO", uint32 version 1,
// KGeoMeta {uint32 W, H; double M, a, Q, Lambda, r_isco, r_disk_in,
// r_disk_out, theta_obs_deg, phi_obs_deg, r_obs} (88 bytes), then W*H
// GeoPixel records {uint8 outcome, uint8 pad[3], float r, redshift, magnif,
// phi_disk, theta_esc, phi_esc} (28 bytes), little-endian.  The layout has
// to match byte for byte so that files move between the reference and this
// renderer.
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/kerrtrace.h"
#include "kt_frame.h"

namespace {

#pragma pack(push, 1)
struct KGeoMeta {
  uint32_t W, H;
  double M_bh, a_bh, Q_bh, Lam;
  double r_isco, r_disk_in, r_disk_out;
  double theta_obs, phi_obs, r_obs;
};
struct GeoPixel {
  uint8_t outcome;
  uint8_t pad[3];
  float r, redshift, magnif, phi_disk, theta_esc, phi_esc;
};
#pragma pack(pop)
static_assert(sizeof(KGeoMeta) == 88, "KGeoMeta is 88 bytes");
static_assert(sizeof(GeoPixel) == 28, "GeoPixel is 28 bytes");

const char kMagic[4] = {'K', 'G', 'E', 'O'};
const uint32_t kVersion = 1;

uint64_t splitmix64(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

kt_status kt_kgeo_write(const char* path, const kt_frame_desc* desc, const kt_geo_soa* g) {
  if (!path || !desc || !g || !g->outcome || !g->r || !g->redshift || !g->magnif || !g->phi_disk ||
      !g->theta_esc || !g->phi_esc)
    return KT_ERR_INVALID_ARGUMENT;
  kt::Frame f;
  kt_frame_derived dv;
  std::string err;
  kt_status st = kt::prepare_frame(desc, &f, &dv, &err);
  if (st != KT_OK) return st;
  KGeoMeta meta;
  meta.W = (uint32_t)desc->width;
  meta.H = (uint32_t)desc->height;
  meta.M_bh = desc->M;
  meta.a_bh = desc->a;
  meta.Q_bh = desc->Q;
  meta.Lam = desc->Lambda;
  meta.r_isco = dv.r_isco;
  meta.r_disk_in = dv.r_disk_in;
  meta.r_disk_out = dv.r_disk_out;
  meta.theta_obs = desc->theta_deg;
  meta.phi_obs = desc->phi_deg;
  meta.r_obs = desc->r_obs;
  FILE* fp = fopen(path, "wb");
  if (!fp) return KT_ERR_IO;
  bool ok = fwrite(kMagic, 1, 4, fp) == 4 && fwrite(&kVersion, 4, 1, fp) == 1 &&
            fwrite(&meta, sizeof meta, 1, fp) == 1;
  const size_t n = (size_t)desc->width * (size_t)desc->height;
  std::vector<GeoPixel> buf(4096);
  for (size_t i0 = 0; ok && i0 < n; i0 += buf.size()) {
    const size_t m = (n - i0 < buf.size()) ? n - i0 : buf.size();
    for (size_t j = 0; j < m; ++j) {
      const size_t i = i0 + j;
      GeoPixel& p = buf[j];
      p.outcome = g->outcome[i];
      p.pad[0] = p.pad[1] = p.pad[2] = 0;
      p.r = (float)g->r[i];
      p.redshift = (float)g->redshift[i];
      p.magnif = (float)g->magnif[i];
      p.phi_disk = (float)g->phi_disk[i];
      p.theta_esc = (float)g->theta_esc[i];
      p.phi_esc = (float)g->phi_esc[i];
    }
    ok = fwrite(buf.data(), sizeof(GeoPixel), m, fp) == m;
  }
  ok = (fclose(fp) == 0) && ok;
  return ok ? KT_OK : KT_ERR_IO;
}

kt_status kt_kgeo_read_header(const char* path, int32_t* width, int32_t* height, double meta10[10]) {
  if (!path || !width || !height) return KT_ERR_INVALID_ARGUMENT;
  FILE* fp = fopen(path, "rb");
  if (!fp) return KT_ERR_IO;
  char magic[4];
  uint32_t ver = 0;
  KGeoMeta meta;
  const bool ok = fread(magic, 1, 4, fp) == 4 && memcmp(magic, kMagic, 4) == 0 &&
                  fread(&ver, 4, 1, fp) == 1 && ver == kVersion &&
                  fread(&meta, sizeof meta, 1, fp) == 1;
  fclose(fp);
  if (!ok || meta.W == 0 || meta.H == 0 || meta.W > 0x7fffffffu || meta.H > 0x7fffffffu ||
      (uint64_t)meta.W * meta.H > 0x7fffffffULL)
    return KT_ERR_IO;
  *width = (int32_t)meta.W;
  *height = (int32_t)meta.H;
  if (meta10) {
    const double v[10] = {meta.M_bh, meta.a_bh, meta.Q_bh, meta.Lam, meta.r_isco,
                          meta.r_disk_in, meta.r_disk_out, meta.theta_obs, meta.phi_obs, meta.r_obs};
    memcpy(meta10, v, sizeof v);
  }
  return KT_OK;
}

kt_status kt_kgeo_read(const char* path, const kt_geo_soa* g, int64_t capacity) {
  int32_t W = 0, H = 0;
  kt_status st = kt_kgeo_read_header(path, &W, &H, nullptr);
  if (st != KT_OK) return st;
  if (!g || !g->outcome || !g->r || !g->redshift || !g->magnif || !g->phi_disk || !g->theta_esc ||
      !g->phi_esc)
    return KT_ERR_INVALID_ARGUMENT;
  const size_t n = (size_t)W * (size_t)H;
  if (capacity < (int64_t)n) return KT_ERR_INVALID_ARGUMENT;
  FILE* fp = fopen(path, "rb");
  if (!fp) return KT_ERR_IO;
  bool ok = fseek(fp, 8 + (long)sizeof(KGeoMeta), SEEK_SET) == 0;
  std::vector<GeoPixel> buf(4096);
  for (size_t i0 = 0; ok && i0 < n; i0 += buf.size()) {
    const size_t m = (n - i0 < buf.size()) ? n - i0 : buf.size();
    ok = fread(buf.data(), sizeof(GeoPixel), m, fp) == m;
    for (size_t j = 0; ok && j < m; ++j) {
      const size_t i = i0 + j;
      const GeoPixel& p = buf[j];
      g->outcome[i] = p.outcome;
      g->r[i] = p.r;
      g->redshift[i] = p.redshift;
      g->magnif[i] = p.magnif;
      g->phi_disk[i] = p.phi_disk;
      g->theta_esc[i] = p.theta_esc;
      g->phi_esc[i] = p.phi_esc;
    }
  }
  fclose(fp);
  return ok ? KT_OK : KT_ERR_IO;
}

// Procedural star field: a dark sky with a faint blue band plus stars whose
// density, brightness and tint come from a splitmix64 stream seeded by
// `seed`.  Integer arithmetic only, so the image is the same on every host.
kt_status kt_starfield(uint64_t seed, int32_t w, int32_t h, uint8_t* rgb) {
  if (w < 1 || h < 1 || !rgb || (int64_t)w * h > ((int64_t)1 << 31)) return KT_ERR_INVALID_ARGUMENT;
  for (int32_t y = 0; y < h; ++y) {
    // Milky-Way-like band around the equator row: brightness falls off with |y - h/2|.
    const int32_t dy = y - h / 2;
    const int32_t band = (int32_t)(24 - (48LL * (dy < 0 ? -dy : dy)) / h);
    for (int32_t x = 0; x < w; ++x) {
      uint64_t s = seed ^ (0x2545f4914f6cdd1dULL * (uint64_t)((int64_t)y * w + x + 1));
      const uint64_t r0 = splitmix64(&s);
      int32_t R = 3, G = 4, B = 10;
      if (band > 0) {
        const int32_t b = band + (int32_t)(r0 & 7);
        R += b / 3;
        G += b / 2;
        B += b;
      }
      const uint32_t pick = (uint32_t)(r0 >> 40) & 0xffffff;  // 24 random bits
      if (pick < 0x24000) {  // ~0.9% of pixels carry a star
        const uint64_t r1 = splitmix64(&s);
        const int32_t lum = 90 + (int32_t)(r1 % 166);
        const int32_t tint = (int32_t)((r1 >> 16) % 3);  // 0 blue-white, 1 white, 2 amber
        R = lum - (tint == 0 ? 25 : 0);
        G = lum - (tint == 2 ? 20 : 0);
        B = lum - (tint == 2 ? 60 : 0);
      }
      uint8_t* p = rgb + 3 * ((size_t)y * w + x);
      p[0] = (uint8_t)(R < 0 ? 0 : R > 255 ? 255 : R);
      p[1] = (uint8_t)(G < 0 ? 0 : G > 255 ? 255 : G);
      p[2] = (uint8_t)(B < 0 ? 0 : B > 255 ? 255 : B);
    }
  }
  return KT_OK;
}

}  // extern "C"
