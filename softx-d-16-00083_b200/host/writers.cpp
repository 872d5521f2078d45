// Output writers: the reference's printI, printPartialI, printI2, printPDF, printPartialPDF and
// printAtoms (IO.cpp:51-167, 273-295), byte for byte, formatted by all host threads.
//
// The reference streams every number through an ofstream set to ios::scientific with the default
// precision 6, i.e. printf's "%.6e".  std::to_chars with chars_format::scientific and precision 6 is
// specified to produce exactly printf's "%.6e" text (correctly rounded, at least two exponent
// digits), so each thread formats a contiguous block of rows into its own buffer and the buffers are
// written in order with one fwrite each.
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "xns_b200.h"

namespace {

inline void put_e(std::string &s, double v) {
  char buf[40];
  const std::to_chars_result r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific, 6);
  s.append(buf, r.ptr);
}

unsigned threads_for(size_t rows) {
  unsigned t = std::max(1u, std::thread::hardware_concurrency());
  return (unsigned)std::min<size_t>(t, std::max<size_t>(1, rows / 4096));
}

// rows [0, n) formatted by row(s, i) into per-thread strings, then written in order
template <class Row>
int write_rows(const char *path, const std::string &head, size_t n, size_t bytes_per_row, Row row) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  const unsigned nt = threads_for(n);
  std::vector<std::string> part(nt);
  auto work = [&](unsigned t) {
    const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
    part[t].reserve((hi - lo) * bytes_per_row);
    for (size_t i = lo; i < hi; i++) row(part[t], i);
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; t++) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  bool ok = head.empty() || fwrite(head.data(), 1, head.size(), f) == head.size();
  for (auto &p : part) ok = ok && fwrite(p.data(), 1, p.size(), f) == p.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? 0 : -1;
}

// printPDF / printPartialPDF: rows up to the last |value| (total) or value (partials) above 1e-10,
// at least one row (IO.cpp:62-64, :88-90)
int write_pdf_rows(const char *path, const double *pdf, uint32_t nhist, double bin, bool by_abs) {
  if (nhist == 0) return -1;
  uint32_t last;
  for (last = nhist - 1; last > 0; last--)
    if ((by_abs ? std::fabs(pdf[last]) : pdf[last]) > 1.e-10) break;
  return write_rows(path, std::string(), (size_t)last + 1, 28, [&](std::string &s, size_t i) {
    put_e(s, ((unsigned int)i + 0.5) * bin);
    s.push_back('\t');
    put_e(s, pdf[i]);
    s.push_back('\n');
  });
}

}  // namespace

extern "C" {

int xns_write_i(const char *path, const double *q, const double *I, uint32_t nq) {
  if (!path || (nq && (!q || !I))) return -1;
  return write_rows(path, std::string(), nq, 28, [&](std::string &s, size_t i) {
    put_e(s, q[i]);
    s.push_back('\t');
    put_e(s, I[i]);
    s.push_back('\n');
  });
}

int xns_write_i2(const char *path, const double *I2D, uint32_t nq, uint32_t nfi) {
  if (!path || (nq && nfi && !I2D)) return -1;
  return write_rows(path, std::string(), nq, 14 * (size_t)nfi + 1, [&](std::string &s, size_t iq) {
    const double *r = I2D + iq * (size_t)nfi;
    for (uint32_t k = 0; k < nfi; k++) {
      put_e(s, r[k]);
      s.push_back('\t');
    }
    s.push_back('\n');
  });
}

int xns_write_pdf(const char *path, const double *pdf, uint32_t nhist, double bin, int partial) {
  if (!path || !pdf) return -1;
  return write_pdf_rows(path, pdf, nhist, bin, !partial);
}

int xns_write_atoms(const char *path, const double *xyz, const uint32_t *n_el, uint32_t nel, const char *const *names) {
  if (!path || !n_el || !names) return -1;
  size_t ntot = 0;
  std::vector<size_t> start(nel + 1, 0);
  for (uint32_t e = 0; e < nel; e++) start[e + 1] = start[e] + n_el[e];
  ntot = start[nel];
  if (ntot && !xyz) return -1;
  // Ntot is an unsigned int in the reference (IO.cpp:277)
  const std::string head = std::to_string((unsigned int)ntot) + "\n\n";
  return write_rows(path, head, ntot, 48, [&](std::string &s, size_t i) {
    const uint32_t e = (uint32_t)(std::upper_bound(start.begin(), start.end(), i) - start.begin()) - 1;
    s.append(names[e]);
    s.push_back(' ');
    put_e(s, xyz[3 * i]);
    s.append("  ");
    put_e(s, xyz[3 * i + 1]);
    s.append("  ");
    put_e(s, xyz[3 * i + 2]);
    s.push_back('\n');
  });
}

}  // extern "C"
