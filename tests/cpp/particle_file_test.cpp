// Host-only checks of the Particles file loader in nbb_simulation.hpp,
// following tests/unit/cpu/particle_file_test.cpp of the reference
// (32/64-bit headers, typed files, truncation, trailing bytes, invalid
// values).  Prints "ok" and exits 0 when every check passes.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "nbb_simulation.hpp"

namespace {

int failures = 0;

void check(bool cond, const std::string &what) {
  if (!cond) {
    std::cerr << "FAILED: " << what << '\n';
    ++failures;
  }
}

struct Data {
  std::vector<double> b[7] = {{1.0, 2.0, 0.0}, {0.1, 0.2, 0.3}, {-1.0, -2.0, -3.0}, {5.0, 6.0, 7.0},
                              {0.5, 0.6, 0.7}, {1.5, 1.6, 1.7}, {-0.5, -0.6, -0.7}};
  std::vector<std::uint8_t> type = {1, 2, 4};
};

void write(const std::string &path, const Data &d, bool header64, bool typed, std::uint64_t count = 3,
           int drop_bytes = 0, bool trailing = false) {
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (header64) {
    out.write(reinterpret_cast<const char *>(&count), 8);
  } else {
    const std::uint32_t c = static_cast<std::uint32_t>(count);
    out.write(reinterpret_cast<const char *>(&c), 4);
  }
  std::string body;
  for (const auto &blk : d.b) body.append(reinterpret_cast<const char *>(blk.data()), blk.size() * 8);
  if (typed) body.append(reinterpret_cast<const char *>(d.type.data()), d.type.size());
  if (drop_bytes) body.resize(body.size() - drop_bytes);
  if (trailing) body.push_back('\x7f');
  out.write(body.data(), static_cast<std::streamsize>(body.size()));
}

std::string error_of(const std::string &path) {
  std::ifstream in(path, std::ios::binary);
  try {
    Particles p(in);
  } catch (const std::runtime_error &e) {
    return e.what();
  }
  return "";
}

}  // namespace

int main(int argc, char **argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  const std::string f = dir + "/particles.bin";
  Data d;
  for (bool h64 : {false, true})
    for (bool typed : {false, true}) {
      write(f, d, h64, typed);
      std::ifstream in(f, std::ios::binary);
      in.seekg(5);  // loading must not depend on the initial stream position
      Particles p(in);
      check(p.size() == 3, "count");
      check(p.x() == d.b[1] && p.vz() == d.b[6] && p.mass() == d.b[0], "blocks");
      check(typed ? p.type() == d.type : p.type() == std::vector<std::uint8_t>(3, 0), "types");
    }
  {
    std::ifstream closed;
    try {
      Particles p(closed);
      check(false, "unopened stream accepted");
    } catch (const std::runtime_error &e) {
      check(std::string(e.what()).find("Invalid or unreadable file stream") != std::string::npos, "unopened");
    }
  }
  { std::ofstream(f, std::ios::binary | std::ios::trunc); }
  check(error_of(f).find("Unsupported particle file layout") != std::string::npos, "empty file");
  write(f, d, false, false, 0, 7 * 3 * 8);
  check(error_of(f).find("Unsupported particle file layout") != std::string::npos, "zero count");
  write(f, d, true, false, 3, 8);
  check(error_of(f).find("Unsupported particle file layout") != std::string::npos, "truncated");
  write(f, d, false, false, 3, 0, true);
  check(error_of(f).find("Unsupported particle file layout") != std::string::npos, "trailing byte");
  Data bad = d;
  bad.type[1] = 255;
  write(f, bad, true, true);
  check(error_of(f).find("Unsupported particle type value") != std::string::npos, "invalid type");
  bad = d;
  bad.b[0][2] = -1.0;
  write(f, bad, true, false);
  check(error_of(f).find("Negative mass value") != std::string::npos, "negative mass");
  bad = d;
  bad.b[0][1] = std::numeric_limits<double>::quiet_NaN();
  write(f, bad, true, false);
  check(error_of(f).find("Non-finite mass value") != std::string::npos, "non-finite mass");
  bad = d;
  bad.b[1][0] = std::numeric_limits<double>::infinity();
  write(f, bad, true, false);
  check(error_of(f).find("Non-finite x position value") != std::string::npos, "non-finite position");
  bad = d;
  bad.b[6][2] = std::numeric_limits<double>::quiet_NaN();
  write(f, bad, true, false);
  check(error_of(f).find("Non-finite z velocity value") != std::string::npos, "non-finite velocity");
  bad = d;
  bad.b[0][0] = 0.0;
  write(f, bad, true, false);
  check(error_of(f).empty(), "zero-mass particle accepted");
  std::remove(f.c_str());
  if (failures) return 1;
  std::cout << "ok\n";
  return 0;
}
