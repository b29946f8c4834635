// restart.cu -- restart files of a handle's device-resident state.
//
// The reference writes a restart as an XML description plus a binary data
// file (solver/actions/WriteRestartFile.cpp:62-90): a <restart> node with the
// attributes version, binary_file, nb_procs, current_time, time_step and
// iteration, and one <field path=... index=...> node per field table; the
// reader (ReadRestartFile.cpp:67-110) checks the version and the process
// count, restores the time and reads each table back.  This file keeps that
// description node and its attributes, and stores each table as raw
// little-endian FP64 rows in the binary file (offset and FNV-1a checksum in
// the field node), so a restart can be read without any CF3 component.
//
// Fields: navier_stokes_solution (N x neq: u, v, [w], p),
// linearized_velocity (N x 4*dim: u_adv, u1, u2, u3), navier_stokes_viscosity
// (N x 1) and, when the handle has one, body_force (N x dim) -- the tables
// that ufem_ns_set_state takes, in the same row layouts -- plus lss_solution
// (N x neq), the linear system's solution vector: the reference keeps it from
// step to step as the next solve's initial guess (NavierStokes.cpp:103 sets
// ZeroLSS reset_solution to false), so it is part of the state a bitwise
// continuation needs.  A restart without it starts from a zero solution, as a
// freshly created reference system would.

#include <cuda_runtime.h>

#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace ufem {
namespace {

struct FieldTable {
  std::string name;
  int64_t rows = 0;
  int cols = 0;
  std::vector<double> data;
};

uint64_t fnv1a(const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

std::string dir_of(const std::string& path) {
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? std::string() : path.substr(0, k + 1);
}

std::string base_of(const std::string& path) {
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? path : path.substr(k + 1);
}

// Value of attribute `key` inside the XML element text `elem` ("" if absent).
std::string attr(const std::string& elem, const std::string& key) {
  const std::string pat = " " + key + "=\"";
  const size_t k = elem.find(pat);
  if (k == std::string::npos) return std::string();
  const size_t b = k + pat.size();
  const size_t e = elem.find('"', b);
  return e == std::string::npos ? std::string() : elem.substr(b, e - b);
}

bool read_file(const std::string& path, std::string& out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char buf[65536];
  size_t n;
  out.clear();
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, n);
  std::fclose(f);
  return true;
}

constexpr char kMagic[8] = {'U', 'F', 'E', 'M', 'R', 'S', 'T', '1'};

}  // namespace
}  // namespace ufem

using namespace ufem;

extern "C" {

int ufem_ns_write_restart(ufem_ns_handle* h, const char* path, double current_time, double time_step,
                          int64_t iteration) {
  if (!h || !path || !*path) return set_error(UFEM_ERR_ARG, "NULL handle or path");
  if (!h->state_set) return set_error(UFEM_ERR_STATE, "write_restart before the state was set");
  const int64_t N = h->N;
  const int d = h->dim, neq = h->neq;
  std::vector<FieldTable> tables(3);
  tables[0] = {"navier_stokes_solution", N, neq, std::vector<double>(size_t(N) * neq)};
  tables[1] = {"linearized_velocity", N, 4 * d, std::vector<double>(size_t(N) * 4 * d)};
  tables[2] = {"navier_stokes_viscosity", N, 1, std::vector<double>(size_t(N))};
  int rc;
  if ((rc = ufem_ns_get_state(h, tables[0].data.data(), tables[1].data.data()))) return rc;
  UFEM_CUDA_TRY(cudaMemcpy(tables[2].data.data(), h->d_nu, size_t(N) * 8, cudaMemcpyDeviceToHost));
  if (h->d_sol) {  // the coupled system's solution vector (a semi-implicit base handle has none)
    FieldTable x{"lss_solution", N, neq, std::vector<double>(size_t(h->nrows))};
    UFEM_CUDA_TRY(cudaMemcpy(x.data.data(), h->d_sol, size_t(h->nrows) * 8, cudaMemcpyDeviceToHost));
    tables.push_back(std::move(x));
  }
  if (h->d_force) {  // padded N x 4 records on the device
    std::vector<double> padded(size_t(N) * 4);
    UFEM_CUDA_TRY(cudaMemcpy(padded.data(), h->d_force, padded.size() * 8, cudaMemcpyDeviceToHost));
    FieldTable f{"body_force", N, d, std::vector<double>(size_t(N) * d)};
    for (int64_t i = 0; i < N; ++i)
      for (int k = 0; k < d; ++k) f.data[size_t(i) * d + k] = padded[size_t(i) * 4 + k];
    tables.push_back(std::move(f));
  }
  const std::string xml_path(path);
  const std::string bin_path = xml_path + ".bin";
  FILE* fb = std::fopen(bin_path.c_str(), "wb");
  if (!fb) return set_error(UFEM_ERR_IO, "cannot open " + bin_path + " for writing");
  bool ok = std::fwrite(kMagic, 1, sizeof(kMagic), fb) == sizeof(kMagic);
  std::vector<int64_t> offsets;
  int64_t off = sizeof(kMagic);
  for (const FieldTable& t : tables) {
    offsets.push_back(off);
    const size_t bytes = t.data.size() * 8;
    ok = ok && std::fwrite(t.data.data(), 1, bytes, fb) == bytes;
    off += int64_t(bytes);
  }
  ok = (std::fclose(fb) == 0) && ok;
  if (!ok) return set_error(UFEM_ERR_IO, "writing " + bin_path + " failed");
  std::string xml = "<?xml version=\"1.0\" encoding=\"ISO-8859-1\"?>\n";
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "<restart version=\"1\" binary_file=\"%s\" nb_procs=\"1\" current_time=\"%.17g\" time_step=\"%.17g\" "
                "iteration=\"%" PRId64 "\" dimension=\"%d\" nodes=\"%" PRId64 "\" elements=\"%" PRId64 "\">\n",
                base_of(bin_path).c_str(), current_time, time_step, iteration, d, N, h->E);
  xml += buf;
  for (size_t k = 0; k < tables.size(); ++k) {
    const FieldTable& t = tables[k];
    std::snprintf(buf, sizeof(buf),
                  "  <field path=\"%s\" index=\"%zu\" rows=\"%" PRId64 "\" cols=\"%d\" offset=\"%" PRId64
                  "\" checksum=\"%016" PRIx64 "\"/>\n",
                  t.name.c_str(), k, t.rows, t.cols, offsets[k], fnv1a(t.data.data(), t.data.size() * 8));
    xml += buf;
  }
  xml += "</restart>\n";
  FILE* fx = std::fopen(xml_path.c_str(), "wb");
  if (!fx) return set_error(UFEM_ERR_IO, "cannot open " + xml_path + " for writing");
  ok = std::fwrite(xml.data(), 1, xml.size(), fx) == xml.size();
  ok = (std::fclose(fx) == 0) && ok;
  if (!ok) return set_error(UFEM_ERR_IO, "writing " + xml_path + " failed");
  return UFEM_OK;
}

int ufem_ns_read_restart(ufem_ns_handle* h, const char* path, double* current_time, double* time_step,
                         int64_t* iteration) {
  if (!h || !path || !*path) return set_error(UFEM_ERR_ARG, "NULL handle or path");
  const std::string xml_path(path);
  std::string xml;
  if (!read_file(xml_path, xml)) return set_error(UFEM_ERR_IO, "cannot read " + xml_path);
  const size_t r0 = xml.find("<restart ");
  if (r0 == std::string::npos) return set_error(UFEM_ERR_IO, "file " + xml_path + " has no restart node");
  const std::string restart = xml.substr(r0, xml.find('>', r0) - r0);
  if (attr(restart, "version") != "1")
    return set_error(UFEM_ERR_IO, "file " + xml_path + " has unsupported version");
  if (attr(restart, "nb_procs") != "1")
    return set_error(UFEM_ERR_IO, "file " + xml_path + " was made for " + attr(restart, "nb_procs") +
                                      " processes, this handle is one process");
  const int64_t N = h->N;
  const int d = h->dim, neq = h->neq;
  if (attr(restart, "nodes") != std::to_string(N) || attr(restart, "dimension") != std::to_string(d))
    return set_error(UFEM_ERR_IO, "restart " + xml_path + " was written for another mesh (nodes or dimension differ)");
  const std::string bin_path = dir_of(xml_path) + attr(restart, "binary_file");
  std::string bin;
  if (!read_file(bin_path, bin)) return set_error(UFEM_ERR_IO, "cannot read " + bin_path);
  if (bin.size() < sizeof(kMagic) || std::memcmp(bin.data(), kMagic, sizeof(kMagic)) != 0)
    return set_error(UFEM_ERR_IO, bin_path + " is not a restart data file");
  std::vector<double> up, lin, nu, force, sol;
  size_t pos = r0;
  while ((pos = xml.find("<field ", pos)) != std::string::npos) {
    const std::string elem = xml.substr(pos, xml.find('>', pos) - pos);
    pos += elem.size();
    const std::string name = attr(elem, "path");
    const int64_t rows = std::strtoll(attr(elem, "rows").c_str(), nullptr, 10);
    const int cols = int(std::strtol(attr(elem, "cols").c_str(), nullptr, 10));
    const int64_t off = std::strtoll(attr(elem, "offset").c_str(), nullptr, 10);
    const uint64_t sum = std::strtoull(attr(elem, "checksum").c_str(), nullptr, 16);
    std::vector<double>* dst = nullptr;
    int want = 0;
    if (name == "navier_stokes_solution") { dst = &up; want = neq; }
    else if (name == "linearized_velocity") { dst = &lin; want = 4 * d; }
    else if (name == "navier_stokes_viscosity") { dst = &nu; want = 1; }
    else if (name == "body_force") { dst = &force; want = d; }
    else if (name == "lss_solution" && h->d_sol) { dst = &sol; want = neq; }
    else return set_error(UFEM_ERR_IO, "restart field " + name + " is not a field of this solver");
    if (rows != N || cols != want) return set_error(UFEM_ERR_IO, "restart field " + name + " has the wrong shape");
    const size_t bytes = size_t(rows) * cols * 8;
    if (off < int64_t(sizeof(kMagic)) || size_t(off) + bytes > bin.size())
      return set_error(UFEM_ERR_IO, "restart field " + name + " lies outside " + bin_path);
    if (fnv1a(bin.data() + off, bytes) != sum)
      return set_error(UFEM_ERR_IO, "restart field " + name + " fails its checksum");
    dst->resize(size_t(rows) * cols);
    std::memcpy(dst->data(), bin.data() + off, bytes);
  }
  if (up.empty() || lin.empty() || nu.empty())
    return set_error(UFEM_ERR_IO, "restart " + xml_path + " lacks the solution, linearized velocity or viscosity");
  int rc;
  if ((rc = ufem_ns_set_state(h, up.data(), lin.data(), nu.data(), force.empty() ? nullptr : force.data())))
    return rc;
  if (h->d_sol && sol.empty())
    UFEM_CUDA_TRY(cudaMemset(h->d_sol, 0, size_t(h->nrows) * 8));
  else if (h->d_sol)
    UFEM_CUDA_TRY(cudaMemcpy(h->d_sol, sol.data(), size_t(h->nrows) * 8, cudaMemcpyHostToDevice));
  h->time = std::strtod(attr(restart, "current_time").c_str(), nullptr);  // Time::current_time
  if (current_time) *current_time = h->time;
  if (time_step) *time_step = std::strtod(attr(restart, "time_step").c_str(), nullptr);
  if (iteration) *iteration = std::strtoll(attr(restart, "iteration").c_str(), nullptr, 10);
  return UFEM_OK;
}

}  // extern "C"
