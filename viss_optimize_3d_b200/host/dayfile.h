// dayfile.h -- binary files of the streaming day loop (host/vissgen_stream_main.cpp),
// replacing the reference's per-day text files (vissgen3d_blockage.cu:309-391)
// and its 6-digit text image (:542-553).  Little-endian; every file is one
// 64-byte header followed by raw arrays:
//
//   offset  0  char[8]  magic   "VISSDAY" / "VISSSKY" / "VISSIMG" (NUL-padded)
//           8  uint32   version (1)
//          12  uint32   bytes per payload element (4 = float32, 8 = float64)
//          16  int64    count   rows (day), pixels (sky, image)
//          24  int64    day     1-based day index (image: first day summed)
//          32  float64  frequency in Hz (0 = not recorded)
//          40  int64    days summed (image; 1 for one day), else 1
//          48  16 bytes zero
//
//   VISSDAY  float32 uvw[n][3], xyza[n][3], xyzb[n][3], bll[n]: the same rows
//            as the text files (unique samples, then their conjugate mirrors;
//            uvw in wavelengths, positions in metres)
//   VISSSKY  float32 B[npix], theta[npix], phi[npix]
//   VISSIMG  image[npix] (float32 per day, float64 for a day sum)
// The payload is exactly count x (elements per item) x element bytes; a file
// of any other size is rejected.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace viss_host {

struct FileHeader {
  char magic[8];
  uint32_t version;
  uint32_t elem_bytes;
  int64_t count;
  int64_t day;
  double frequency;
  int64_t days;
  int64_t reserved[2];
};
static_assert(sizeof(FileHeader) == 64, "64-byte header");

constexpr uint32_t kFileVersion = 1;
constexpr int kDayFloatsPerRow = 10;  // uvw 3 + xyza 3 + xyzb 3 + bll 1
constexpr int kSkyFloatsPerPixel = 3;

inline FileHeader make_header(const char *magic, uint32_t elem_bytes, int64_t count, int64_t day,
                              double frequency, int64_t days) {
  FileHeader h;
  std::memset(&h, 0, sizeof(h));
  std::strncpy(h.magic, magic, sizeof(h.magic));
  h.version = kFileVersion;
  h.elem_bytes = elem_bytes;
  h.count = count;
  h.day = day;
  h.frequency = frequency;
  h.days = days;
  return h;
}

// Opens `path`, reads and checks the header against `magic` and the expected
// payload (items x per_item elements).  On success the file is positioned at
// the payload; on failure returns nullptr with a message in `err`.
inline std::FILE *open_checked(const std::string &path, const char *magic, int per_item,
                               FileHeader &h, std::string &err) {
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open " + path;
    return nullptr;
  }
  if (std::fread(&h, sizeof(h), 1, f) != 1 || std::strncmp(h.magic, magic, 8) != 0 ||
      h.version != kFileVersion || (h.elem_bytes != 4 && h.elem_bytes != 8) || h.count < 0) {
    err = path + ": not a version-1 " + magic + " file";
    std::fclose(f);
    return nullptr;
  }
  std::fseek(f, 0, SEEK_END);
  const long long size = std::ftell(f);
  const long long want =
      static_cast<long long>(sizeof(h)) + h.count * static_cast<long long>(per_item) * h.elem_bytes;
  if (size != want) {
    err = path + ": size " + std::to_string(size) + " bytes, header says " + std::to_string(want);
    std::fclose(f);
    return nullptr;
  }
  std::fseek(f, sizeof(h), SEEK_SET);
  return f;
}

inline bool write_file(const std::string &path, const FileHeader &h, const void *payload,
                       size_t bytes) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  if (ok && bytes) ok = std::fwrite(payload, 1, bytes, f) == bytes;
  return std::fclose(f) == 0 && ok;
}

}  // namespace viss_host
