// The host half of the device's surface text (gvh_surface_host.cpp: format_rows with a
// DeviceText): the device's text of the rows the fast %g formats, plus the rows it leaves to
// the exact path (HostRow: values, row index, text offset), must give the same text as
// formatting every row on the host, in order, for any pool size and any mix of the two.
// Built with the host compiler from gvh_surface_host.cpp; prints "<n> mismatches".
#include <stdio.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "gvh_format.hpp"
#include "gvh_surface_internal.h"

using namespace gvh;
using namespace gvh::surface;

namespace {

std::string row_text(const double *v) {
  char buf[kColumns * 32];
  char *p = buf;
  for (int k = 0; k < kColumns; ++k) {
    p = fmt::g6(p, buf + sizeof buf, v[k]);
    *p++ = k + 1 < kColumns ? ' ' : '\n';
  }
  return std::string(buf, p - buf);
}

// The device's side: text of the rows whose every number the fast path formats, host rows
// for the others (in shuffled order, as the device's atomics leave them, then sorted by row
// as find_end sorts them).
void device_side(const std::vector<double> &rows, long long n, std::string &text, std::vector<HostRow> &host,
                 std::mt19937_64 &rng) {
  text.clear();
  host.clear();
  for (long long r = 0; r < n; ++r) {
    const double *v = rows.data() + r * kColumns;
    char buf[kColumns * 32];
    char *p = buf;
    bool fast = true;
    for (int k = 0; k < kColumns && fast; ++k) {
      char *q = fmt::g6_fast(p, v[k]);
      if (!q) {
        fast = false;
        break;
      }
      p = q;
      *p++ = k + 1 < kColumns ? ' ' : '\n';
    }
    if (fast) {
      text.append(buf, p - buf);
    } else {
      HostRow h;
      h.text_off = (long long)text.size();
      h.row = r;
      for (int k = 0; k < kColumns; ++k) h.v[k] = v[k];
      host.push_back(h);
    }
  }
  std::shuffle(host.begin(), host.end(), rng);
  std::sort(host.begin(), host.end(), [](const HostRow &a, const HostRow &b) { return a.row < b.row; });
}

// Rows with a share of numbers outside the fast path's range (|x| ~ 1e-28, 1e30), placed by
// `pattern`: 0 none, 1 every row, 2 random rows, 3 runs at the start and the end.
std::vector<double> make_rows(long long n, int pattern, std::mt19937_64 &rng) {
  std::uniform_real_distribution<double> u(-3.0, 3.0);
  std::vector<double> rows((size_t)n * kColumns);
  for (auto &x : rows) x = u(rng) * pow(10.0, (double)(int)(u(rng) * 2));
  for (long long r = 0; r < n; ++r) {
    bool odd = pattern == 1 || (pattern == 2 && rng() % 7 == 0) ||
               (pattern == 3 && (r < 3 || r >= n - 3 || (r > n / 2 && r < n / 2 + 5)));
    if (odd) rows[(size_t)r * kColumns + (size_t)(rng() % kColumns)] = (rng() & 1) ? 1.7e-28 : -4.2e30;
  }
  return rows;
}

}  // namespace

int main() {
  std::mt19937_64 rng(12345);
  long long mismatches = 0, cases = 0;
  const long long sizes[] = {1, 2, 7, 300, 20000, 60000};
  for (int threads : {1, 3, 8}) {
    Pool pool(threads);
    for (long long n : sizes)
      for (int pattern = 0; pattern < 4; ++pattern)
        for (int keep_rows = 0; keep_rows < 2; ++keep_rows) {
          const std::vector<double> rows = make_rows(n, pattern, rng);
          std::string text;
          std::vector<HostRow> host;
          device_side(rows, n, text, host, rng);
          std::string expect;
          for (long long r = 0; r < n; ++r) expect += row_text(rows.data() + r * kColumns);
          DeviceText dt;
          dt.text = text.data();
          dt.bytes = (long long)text.size();
          dt.host_rows = host.data();
          dt.n_host = (long long)host.size();
          int calls = 0;
          dt.ready = [&calls] { __atomic_add_fetch(&calls, 1, __ATOMIC_RELAXED); };
          Result out;
          const int outputs = OUT_TEXT | (keep_rows ? OUT_ROWS : 0);
          format_rows(keep_rows ? rows.data() : nullptr, n, pool, outputs, out, pattern & 1, dt);
          if (pattern & 1) pool.wait();
          ++cases;
          bool ok = out.text() == expect && out.elements == n && calls == (int)out.parts.size();
          if (keep_rows) {
            std::vector<double> got;
            for (auto &p : out.parts) got.insert(got.end(), p.rows.begin(), p.rows.end());
            ok = ok && got == rows;
          }
          if (!ok) {
            ++mismatches;
            printf("mismatch: threads %d n %lld pattern %d keep_rows %d (host rows %zu, parts %zu)\n", threads, n,
                   pattern, keep_rows, host.size(), out.parts.size());
          }
        }
  }
  printf("%lld cases, %lld mismatches\n", cases, mismatches);
  return mismatches ? 1 : 0;
}
