// Point-cloud output of the fused depth maps: binary little-endian PLY in the layout of the reference's dense output
// (crates/dense/src/densify.rs:143-153 -> crates/core/src/io/ply.rs:82-140 with PlyLayout::XyzNormalRgb):
// "x y z nx ny nz red green blue", type names float / uchar, 27 bytes per point (15 without normals; colour 255 when
// none is given).
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/patchstereo.h"

extern "C" int ps_write_ply(const char* path, uint64_t n, const float* positions, const float* normals,
                            const uint8_t* colors) {
  if (!path || (n && !positions)) return PS_EINVAL;
  FILE* f = fopen(path, "wb");
  if (!f) return PS_EINVAL;
  std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
  h += "property float x\nproperty float y\nproperty float z\n";
  if (normals) h += "property float nx\nproperty float ny\nproperty float nz\n";
  h += "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n";
  bool ok = fwrite(h.data(), 1, h.size(), f) == h.size();
  const size_t rec = 12 + (normals ? 12 : 0) + 3;
  std::vector<uint8_t> buf;
  buf.reserve(rec * 65536);
  const uint8_t white[3] = {255, 255, 255};
  for (uint64_t i = 0; i < n && ok; ++i) {
    const uint8_t* p = (const uint8_t*)(positions + 3 * i);  // IEEE binary32, little-endian host
    buf.insert(buf.end(), p, p + 12);
    if (normals) {
      const uint8_t* q = (const uint8_t*)(normals + 3 * i);
      buf.insert(buf.end(), q, q + 12);
    }
    const uint8_t* c = colors ? colors + 3 * i : white;
    buf.insert(buf.end(), c, c + 3);
    if (buf.size() >= rec * 65536) {
      ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
      buf.clear();
    }
  }
  if (ok && !buf.empty()) ok = fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? PS_OK : PS_EINVAL;
}
