// Reader for the *_tb.dat layout of src/wannier_tb.cpp:15-113.
//
// Line structure: comment; three lattice rows; num_wann; nrpts; (nrpts-1)/15+1 degeneracy lines;
// one separator line; per R cell an "n1 n2 n3" line, nw^2 lines "m n Re Im", one separator line;
// then per R cell (same order) a header line and nw^2 lines "m n xRe xIm yRe yIm zRe zIm", one
// separator line.  The element of line "m n" is stored at [n-1][m-1] (src/wannier_tb.cpp:73-74,
// 101-102).  Unlike the reference, malformed files raise an error instead of reading garbage.
#include "tb_model.hpp"

#include <charconv>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace hhg {
namespace {

struct LineReader {
  std::ifstream in;
  std::string path;
  int lineno = 0;
  std::string next(const char* what) {
    std::string line;
    if (!std::getline(in, line)) {
      std::ostringstream os;
      os << "TB file " << path << ": unexpected end of file while reading " << what << " (line " << lineno + 1
         << ")";
      throw std::runtime_error(os.str());
    }
    ++lineno;
    return line;
  }
  [[noreturn]] void fail(const std::string& msg) {
    std::ostringstream os;
    os << "TB file " << path << " line " << lineno << ": " << msg;
    throw std::runtime_error(os.str());
  }
};

// Numbers of one line, read with strtol / strtod semantics (the conversions istream's operator>> uses,
// so the values are the same; a per-line istringstream made setup parse-bound for large models).
// Decimal reals go through std::from_chars, which like strtod rounds correctly (the same double, in the
// "C" locale the library runs in) and is several times faster; anything it declines (a leading '+',
// hexadecimal, out of range) falls back to strtod.
struct Fields {
  const char* p;
  const char* endl;
  bool ok = true;
  explicit Fields(const std::string& s) : p(s.c_str()), endl(s.c_str() + s.size()) {}
  long integer() {
    char* end = nullptr;
    const long v = std::strtol(p, &end, 10);
    ok = ok && end != p;
    p = end;
    return v;
  }
  double real() {
    const char* q = p;
    while (q < endl && (*q == ' ' || *q == '\t' || *q == '\r' || *q == '\n' || *q == '\v' || *q == '\f')) ++q;
    double v = 0.0;
    const auto res = std::from_chars(q, endl, v, std::chars_format::general);
    if (res.ec == std::errc() && res.ptr != q && (res.ptr == endl || (*res.ptr != 'x' && *res.ptr != 'X'))) {
      p = res.ptr;
      return v;
    }
    char* end = nullptr;
    v = std::strtod(p, &end);
    ok = ok && end != p;
    p = end;
    return v;
  }
};

}  // namespace

TBModel parse_tb(const std::string& path) {
  LineReader rd;
  rd.path = path;
  rd.in.open(path);
  if (!rd.in) throw std::runtime_error("Error opening wannier tb file: " + path);
  TBModel m;
  m.comment = rd.next("comment");
  for (int i = 0; i < 3; ++i) {
    std::istringstream is(rd.next("lattice vectors"));
    if (!(is >> m.lattice[i][0] >> m.lattice[i][1] >> m.lattice[i][2])) rd.fail("bad lattice vector");
  }
  {
    std::istringstream is(rd.next("num_wann"));
    if (!(is >> m.nw) || m.nw <= 0) rd.fail("bad number of orbitals");
  }
  {
    std::istringstream is(rd.next("nrpts"));
    if (!(is >> m.nsites) || m.nsites <= 0) rd.fail("bad number of R cells");
  }
  const int ndeg = (m.nsites - 1) / 15 + 1;
  for (int i = 0; i < ndeg; ++i) {
    std::istringstream is(rd.next("degeneracies"));
    int d;
    while (is >> d) m.degeneracy.push_back(d);
  }
  rd.next("separator");
  const int nw = m.nw, nw2 = nw * nw;
  m.R.assign((size_t)m.nsites * 3, 0);
  m.hop.assign((size_t)m.nsites * nw2, cd(0, 0));
  for (int a = 0; a < 3; ++a) m.bc[a].assign((size_t)m.nsites * nw2, cd(0, 0));
  for (int s = 0; s < m.nsites; ++s) {
    {
      const std::string line = rd.next("R cell");
      Fields f(line);
      for (int a = 0; a < 3; ++a) m.R[3 * s + a] = (int)f.integer();
      if (!f.ok) rd.fail("bad R cell line");
    }
    for (int q = 0; q < nw2; ++q) {
      const std::string line = rd.next("hopping");
      Fields f(line);
      const long o1 = f.integer(), o2 = f.integer();
      const double re = f.real(), im = f.real();
      if (!f.ok || o1 < 1 || o1 > nw || o2 < 1 || o2 > nw) rd.fail("bad hopping line");
      m.hop[(size_t)s * nw2 + (o2 - 1) * nw + (o1 - 1)] = cd(re, im);
    }
    rd.next("separator");
  }
  for (int s = 0; s < m.nsites; ++s) {
    rd.next("position block header");
    for (int q = 0; q < nw2; ++q) {
      const std::string line = rd.next("position element");
      Fields f(line);
      const long o1 = f.integer(), o2 = f.integer();
      double v[6];
      for (double& x : v) x = f.real();
      if (!f.ok || o1 < 1 || o1 > nw || o2 < 1 || o2 > nw) rd.fail("bad position line");
      for (int a = 0; a < 3; ++a) m.bc[a][(size_t)s * nw2 + (o2 - 1) * nw + (o1 - 1)] = cd(v[2 * a], v[2 * a + 1]);
    }
    std::string sep;
    if (std::getline(rd.in, sep)) ++rd.lineno;  // the last separator may be missing
  }
  return m;
}

}  // namespace hhg
