// RSF (Madagascar regularly sampled format) files: the I/O boundary of the
// reference's tools (src/tool/main-*.cpp read velocities and shots and
// write shots and models through sf_input / sf_output), written afresh.
//
// A header is text: whitespace-separated key=value tokens (values may be
// double-quoted), any number per line, later lines overriding earlier ones
// (Madagascar appends each program's parameters to the history).  in=
// names the binary file; in="stdin" means the binary follows the header
// after the bytes 0x0c 0x0c 0x04.  Data are native little-endian float32
// (esize=4, data_format="native_float"), axis 1 fastest.
//
// Layouts used by the reference:
//   velocity: n1 = nz, n2 = nx           -> vel[ix][iz] (x-major, z contiguous)
//   shots:    n1 = nt, n2 = ng, n3 = ns  -> on disk [is][ig][it]; the
//             reference transposes each shot to [it][ig] on reading
//             (shotdata-reader.cpp:54-64) and back on writing.
// Host code only; nothing here touches the GPU.
#include <cctype>
#include <cstdio>
#include <iterator>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "common.hpp"

namespace swfwi {
namespace {

struct Header {
  std::map<std::string, std::string> kv;
  std::string path;            // the header file
  long long embedded_at = -1;  // offset of embedded binary (in="stdin")
};

const char kEmbedMark[3] = {0x0c, 0x0c, 0x04};

Header parse_header(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw Error(SWFWI_ERR_BAD_ARG, "cannot open RSF header " + path);
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  Header h;
  h.path = path;
  size_t end = text.size();
  for (size_t i = 0; i + 2 < text.size(); i++)
    if (text[i] == kEmbedMark[0] && text[i + 1] == kEmbedMark[1] && text[i + 2] == kEmbedMark[2]) {
      end = i;
      h.embedded_at = (long long)i + 3;
      break;
    }
  // tokens: key=value with an optional "quoted value"
  size_t i = 0;
  while (i < end) {
    while (i < end && std::isspace((unsigned char)text[i])) i++;
    size_t s = i;
    bool quoted = false;
    while (i < end && (quoted || !std::isspace((unsigned char)text[i]))) {
      if (text[i] == '"') quoted = !quoted;
      i++;
    }
    std::string tok = text.substr(s, i - s);
    size_t eq = tok.find('=');
    if (eq == std::string::npos || eq == 0) continue;
    std::string key = tok.substr(0, eq), val = tok.substr(eq + 1);
    if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
    h.kv[key] = val;
  }
  return h;
}

bool get(const Header &h, const std::string &k, std::string &v) {
  auto it = h.kv.find(k);
  if (it == h.kv.end()) return false;
  v = it->second;
  return true;
}

std::string dir_of(const std::string &p) {
  size_t s = p.find_last_of('/');
  return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

// The binary: file name and byte offset of element 0.
void data_location(const Header &h, std::string &file, long long &offset) {
  std::string in;
  if (!get(h, "in", in)) throw Error(SWFWI_ERR_BAD_ARG, "RSF header has no in= : " + h.path);
  std::string fmt = "native_float", es = "4";
  get(h, "data_format", fmt);
  get(h, "esize", es);
  if (fmt != "native_float" || es != "4")
    throw Error(SWFWI_ERR_BAD_ARG, "only native_float RSF data are supported: " + h.path);
  if (in == "stdin") {
    if (h.embedded_at < 0) throw Error(SWFWI_ERR_BAD_ARG, "in=stdin without embedded data: " + h.path);
    file = h.path;
    offset = h.embedded_at;
    return;
  }
  std::ifstream t(in, std::ios::binary);
  if (t) {
    file = in;
  } else {
    file = dir_of(h.path) + "/" + in;   // a path relative to the header's folder
    std::ifstream t2(file, std::ios::binary);
    if (!t2) throw Error(SWFWI_ERR_BAD_ARG, "cannot open RSF data " + in);
  }
  offset = 0;
}

long long count_of(const Header &h) {
  long long n = 1;
  for (int a = 1; a <= 9; a++) {
    std::string v;
    if (get(h, "n" + std::to_string(a), v)) n *= std::stoll(v);
  }
  return n;
}

void read_floats(const Header &h, float *out, long long count, long long first) {
  std::string file;
  long long off;
  data_location(h, file, off);
  std::ifstream f(file, std::ios::binary);
  if (!f) throw Error(SWFWI_ERR_BAD_ARG, "cannot open RSF data " + file);
  f.seekg(off + first * 4);
  f.read(reinterpret_cast<char *>(out), count * 4);
  if (f.gcount() != count * 4) throw Error(SWFWI_ERR_BAD_ARG, "RSF data shorter than its header says: " + file);
}

void write_file(const std::string &header, const std::string &data_path, const float *data, long long count,
                const std::string &keys) {
  const std::string dp = data_path.empty() ? header + "@" : data_path;
  {
    std::ofstream d(dp, std::ios::binary | std::ios::trunc);
    if (!d) throw Error(SWFWI_ERR_BAD_ARG, "cannot write RSF data " + dp);
    d.write(reinterpret_cast<const char *>(data), count * 4);
    if (!d) throw Error(SWFWI_ERR_BAD_ARG, "short write to " + dp);
  }
  std::ofstream f(header, std::ios::trunc);
  if (!f) throw Error(SWFWI_ERR_BAD_ARG, "cannot write RSF header " + header);
  f << "swfwi_b200\n" << keys << "\tin=\"" << dp << "\"\n\tesize=4\n\tdata_format=\"native_float\"\n";
  if (!f) throw Error(SWFWI_ERR_BAD_ARG, "short write to " + header);
}

std::string axis_keys(int ndim, const int *n, const float *d, const float *o) {
  std::ostringstream s;
  s.precision(9);
  for (int a = 0; a < ndim; a++) {
    s << "\tn" << a + 1 << "=" << n[a] << "\n";
    if (d) s << "\td" << a + 1 << "=" << d[a] << "\n";
    if (o) s << "\to" << a + 1 << "=" << o[a] << "\n";
  }
  return s.str();
}

}  // namespace
}  // namespace swfwi

using namespace swfwi;

extern "C" {

int swfwi_rsf_get(const char *path, const char *key, char *value, int len) {
  return guarded([&] {
    SWFWI_REQUIRE(path && key && value && len > 0, "bad arguments");
    Header h = parse_header(path);
    std::string v;
    if (!get(h, key, v)) throw Error(SWFWI_ERR_BAD_ARG, std::string("RSF header has no ") + key);
    SWFWI_REQUIRE((int)v.size() < len, "value longer than the buffer");
    std::memcpy(value, v.c_str(), v.size() + 1);
  });
}

int swfwi_rsf_dims(const char *path, int *ndim, int *n, float *d, float *o) {
  return guarded([&] {
    SWFWI_REQUIRE(path && ndim && n, "bad arguments");
    Header h = parse_header(path);
    int nd = 0;
    for (int a = 1; a <= 9; a++) {
      std::string v;
      n[a - 1] = get(h, "n" + std::to_string(a), v) ? std::stoi(v) : 1;
      if (d) d[a - 1] = get(h, "d" + std::to_string(a), v) ? std::stof(v) : 1.0f;
      if (o) o[a - 1] = get(h, "o" + std::to_string(a), v) ? std::stof(v) : 0.0f;
      if (n[a - 1] > 1) nd = a;
    }
    *ndim = nd;
  });
}

int swfwi_rsf_read(const char *path, float *out, long long count, long long first) {
  return guarded([&] {
    SWFWI_REQUIRE(path && out && count >= 0 && first >= 0, "bad arguments");
    Header h = parse_header(path);
    SWFWI_REQUIRE(first + count <= count_of(h), "read beyond the RSF dimensions");
    read_floats(h, out, count, first);
  });
}

int swfwi_rsf_write(const char *path, const char *data_path, const float *data, int ndim, const int *n,
                    const float *d, const float *o, const char *extra) {
  return guarded([&] {
    SWFWI_REQUIRE(path && data && ndim >= 1 && ndim <= 9 && n, "bad arguments");
    long long count = 1;
    for (int a = 0; a < ndim; a++) {
      SWFWI_REQUIRE(n[a] >= 1, "axis lengths must be positive");
      count *= n[a];
    }
    std::string keys = axis_keys(ndim, n, d, o);
    if (extra) keys += extra;
    write_file(path, data_path ? data_path : "", data, count, keys);
  });
}

int swfwi_rsf_read_shots(const char *path, float *dobs, int ns, int nt, int ng) {
  return guarded([&] {
    SWFWI_REQUIRE(path && dobs && ns > 0 && nt > 0 && ng > 0, "bad arguments");
    Header h = parse_header(path);
    SWFWI_REQUIRE((long long)ns * nt * ng <= count_of(h), "shot file smaller than ns*nt*ng");
    std::vector<float> trace((size_t)nt * ng);
    for (int is = 0; is < ns; is++) {
      read_floats(h, trace.data(), (long long)nt * ng, (long long)is * nt * ng);
      float *dst = dobs + (size_t)is * nt * ng;
      for (int ig = 0; ig < ng; ig++)        // matrix_transpose(trace, dst, nt, ng)
        for (int it = 0; it < nt; it++) dst[(size_t)it * ng + ig] = trace[(size_t)ig * nt + it];
    }
  });
}

int swfwi_rsf_write_shots(const char *path, const char *data_path, const float *dobs, int ns, int nt, int ng,
                          float dt, float dgx, const char *extra) {
  return guarded([&] {
    SWFWI_REQUIRE(path && dobs && ns > 0 && nt > 0 && ng > 0, "bad arguments");
    std::vector<float> disk((size_t)ns * nt * ng);
    for (int is = 0; is < ns; is++) {
      const float *src = dobs + (size_t)is * nt * ng;
      float *dst = disk.data() + (size_t)is * nt * ng;
      for (int it = 0; it < nt; it++)
        for (int ig = 0; ig < ng; ig++) dst[(size_t)ig * nt + it] = src[(size_t)it * ng + ig];
    }
    const int n[3] = {nt, ng, ns};
    const float d[3] = {dt, dgx, 1.0f}, o[3] = {0.0f, 0.0f, 0.0f};
    std::string keys = axis_keys(3, n, d, o);
    keys += "\tlabel1=\"Time\"\n\tlabel2=\"Lateral\"\n\tlabel3=\"Shot\"\n\tunit1=\"sec\"\n\tunit2=\"m\"\n";
    if (extra) keys += extra;
    write_file(path, data_path ? data_path : "", disk.data(), (long long)disk.size(), keys);
  });
}

}  // extern "C"
