// Mutation check of the beam-file readers (bmad-ecosystem_b200/csrc/h5beam.cpp, beamio.cpp), built
// with AddressSanitizer and UBSan by tests/test_beamio_hdf5_cpu.py: random bytes of a valid file are
// overwritten (and the file sometimes truncated); every read, and every append of a bunch to such a
// file, must end with a status code, never with an access outside the file's bytes.
// Usage: beamfile_fuzz hdf5|ascii|append <file> <seed> <iterations> <tmp>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/bmadgpu.h"

int main(int argc, char** argv) {
  if (argc != 6) return 2;
  const bool hdf5 = std::strcmp(argv[1], "hdf5") == 0, append = std::strcmp(argv[1], "append") == 0;
  argv++;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::vector<unsigned char> src;
  for (int c; (c = std::fgetc(f)) != EOF;) src.push_back((unsigned char)c);
  std::fclose(f);
  std::mt19937_64 rng(std::strtoull(argv[2], nullptr, 10));
  const int iters = std::atoi(argv[3]);
  bmadgpu_param p{};
  p.mass = 0.51099895069e6;
  p.p0c = 1e9;
  p.charge = 1;
  int ok = 0, err = 0;
  for (int it = 0; it < iters; it++) {
    std::vector<unsigned char> d = src;
    const int n_mut = 1 + (int)(rng() % 8);
    for (int k = 0; k < n_mut; k++) d[rng() % d.size()] = (unsigned char)(rng() % 256);
    if (rng() % 4 == 0) d.resize(rng() % d.size());
    FILE* o = std::fopen(argv[4], "wb");
    if (!o) return 2;
    std::fwrite(d.data(), 1, d.size(), o);
    std::fclose(o);
    int64_t n = 0;
    int32_t nb = 0;
    if (append) {
      std::vector<double> vec(30, 1e-3), beta(5, 0.99), t(5, 0.0);
      std::vector<int32_t> st(5, 1), ie(5, 0), loc(5, 2);
      bmadgpu_bunch b{5, vec.data(), beta.data(), t.data(), st.data(), ie.data(), nullptr, loc.data()};
      int rc = bmadgpu_beam_write_hdf5(argv[4], &b, &p, 0.0, BMADGPU_BEAM_APPEND);
      if (rc == 0) rc = bmadgpu_beam_read_hdf5(argv[4], &p, 0, 0, nullptr, &n, &nb);
      (rc == 0 ? ok : err)++;
      continue;
    }
    int rc = hdf5 ? bmadgpu_beam_read_hdf5(argv[4], &p, 0, 0, nullptr, &n, &nb)
                  : bmadgpu_beam_read_ascii(argv[4], &p, nullptr, &n);
    if (rc == 0 && n > 0 && n < 100000) {
      std::vector<double> vec(6 * n), beta(n), t(n);
      std::vector<int32_t> st(n), ie(n), loc(n);
      bmadgpu_bunch b{n, vec.data(), beta.data(), t.data(), st.data(), ie.data(), nullptr, loc.data()};
      rc = hdf5 ? bmadgpu_beam_read_hdf5(argv[4], &p, 0, 0, &b, &n, &nb) : bmadgpu_beam_read_ascii(argv[4], &p, &b, &n);
    }
    (rc == 0 ? ok : err)++;
  }
  std::printf("read %d, refused %d\n", ok, err);
  return 0;
}
