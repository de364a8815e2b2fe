// checkpoint.h — the file format of the solver's auto-save (params.auto_save)
// and of hprqp_solve_resume.
//
// The reference writes an HDF5 file (save_state_to_hdf5!,
// src/algorithm.jl:183-301) with the datasets current/..., best/... and
// parameters/....  HDF5 is not available to this library, so the same
// datasets go into a plain binary container of named arrays:
//
//   "HPRQPCK1"                                   8-byte magic
//   repeated to the end of the file:
//     u16 name length, name bytes                e.g. "current/x_org"
//     u8  type                                   1 = f64, 2 = i64, 3 = string
//     u64 count                                  elements (bytes for a string)
//     payload                                    little-endian
//
// A "resume/..." section beside them holds the scaled working state the
// method needs to continue (hprqp_solve_resume).  The writer fills
// `<path>.tmp` and renames it over `<path>`, so a reader never sees a
// half-written file.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace hprqp {
namespace ck {

constexpr char kMagic[9] = "HPRQPCK1";
enum : uint8_t { kF64 = 1, kI64 = 2, kStr = 3 };

struct Writer {
  std::string buf = std::string(kMagic, 8);
  void head(const std::string& name, uint8_t type, uint64_t count) {
    const uint16_t len = (uint16_t)name.size();
    buf.append((const char*)&len, 2);
    buf.append(name);
    buf.push_back((char)type);
    buf.append((const char*)&count, 8);
  }
  void f64(const std::string& name, const double* v, int64_t count) {
    head(name, kF64, (uint64_t)count);
    if (count > 0) buf.append((const char*)v, sizeof(double) * (size_t)count);
  }
  void f64(const std::string& name, double v) { f64(name, &v, 1); }
  void i64(const std::string& name, int64_t v) {
    head(name, kI64, 1);
    buf.append((const char*)&v, 8);
  }
  void str(const std::string& name, const std::string& s) {
    head(name, kStr, (uint64_t)s.size());
    buf.append(s);
  }
  // false (and `err` set) when the file cannot be written
  bool write(const std::string& path, std::string& err) const {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) {
      err = "cannot open " + tmp + " for writing";
      return false;
    }
    const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) {
      std::remove(tmp.c_str());
      err = "short write to " + tmp;
      return false;
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
      std::remove(tmp.c_str());
      err = "cannot rename " + tmp + " to " + path;
      return false;
    }
    return true;
  }
};

struct Record {
  uint8_t type = 0;
  std::vector<double> f;
  std::vector<int64_t> i;
  std::string s;
};

struct Reader {
  std::map<std::string, Record> recs;
  // false (and `err` set) on a missing, foreign or truncated file
  bool read(const std::string& path, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
      err = "cannot open checkpoint " + path;
      return false;
    }
    std::string all;
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) all.append(chunk, got);
    std::fclose(f);
    if (all.size() < 8 || std::memcmp(all.data(), kMagic, 8) != 0) {
      err = path + " is not a libhprqp checkpoint";
      return false;
    }
    size_t at = 8;
    auto take = [&](void* dst, size_t len) {
      if (at + len > all.size()) return false;
      std::memcpy(dst, all.data() + at, len);
      at += len;
      return true;
    };
    while (at < all.size()) {
      uint16_t len = 0;
      uint8_t type = 0;
      uint64_t count = 0;
      if (!take(&len, 2)) break;
      std::string name(len, '\0');
      if (!take(&name[0], len) || !take(&type, 1) || !take(&count, 8)) {
        err = "truncated checkpoint " + path;
        return false;
      }
      Record r;
      r.type = type;
      const size_t width = type == kStr ? 1 : 8;
      if (count > (all.size() - at) / width) {
        err = "truncated checkpoint " + path;
        return false;
      }
      if (type == kF64) {
        r.f.resize(count);
        take(r.f.data(), 8 * count);
      } else if (type == kI64) {
        r.i.resize(count);
        take(r.i.data(), 8 * count);
      } else if (type == kStr) {
        r.s.resize(count);
        take(&r.s[0], count);
      } else {
        err = "unknown record type in " + path;
        return false;
      }
      recs[name] = std::move(r);
    }
    return true;
  }
  const Record* get(const std::string& name) const {
    auto it = recs.find(name);
    return it == recs.end() ? nullptr : &it->second;
  }
};

}  // namespace ck
}  // namespace hprqp
