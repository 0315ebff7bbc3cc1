// .dg state files, byte-compatible with the reference's write_state /
// read_state (io.cpp:33-159): u64 tstep, u64 nx ny nz, u64 p q, s64 bounds[6],
// u64 noutput, f64 nodes[E (q+1)^3 3], then per output u64 keylen, key bytes,
// f64 data[E 5 (p+1)^3].  Outputs are written in the order the reference's
// hash map iterates them: djb2 bucket (mod 256) ascending, insertion order
// within a bucket, a repeated key replacing the earlier one
// (data_structures.cpp:444-463, 538-583).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dgb200.h"

namespace {

uint32_t djb2(const char* s)
{
  uint32_t h = 5381;
  for (; *s; ++s) h = h * 33 + (uint32_t)(int)*s;
  return h;
}

struct File {
  FILE* f;
  explicit File(FILE* f_) : f(f_) {}
  ~File()
  {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" int dgb_write_state(const char* fname, unsigned long long tstep, const dgb_mesh_desc* m,
                               int noutput, const char* const* keys, const double* const* data)
{
  if (!fname || !m || !m->nodes || noutput < 0 || (noutput > 0 && (!keys || !data))) return DGB_ERR_ARG;
  const uint64_t E = (uint64_t)m->nx * m->ny * m->nz;
  const uint64_t nq = (uint64_t)(m->q + 1) * (m->q + 1) * (m->q + 1);
  const uint64_t nb = (uint64_t)(m->p + 1) * (m->p + 1) * (m->p + 1);
  // hash-map iteration order with replacement of repeated keys
  std::vector<std::vector<int>> bucket(256);
  for (int o = 0; o < noutput; ++o) {
    std::vector<int>& b = bucket[djb2(keys[o]) % 256];
    bool replaced = false;
    for (int& k : b)
      if (strcmp(keys[k], keys[o]) == 0) {
        k = o;
        replaced = true;
      }
    if (!replaced) b.push_back(o);
  }
  std::vector<int> order;
  for (auto& b : bucket)
    for (int k : b) order.push_back(k);
  File fp(fopen(fname, "wb"));
  if (!fp.f) return DGB_ERR_IO;
  const uint64_t hdr[6] = {tstep, (uint64_t)m->nx, (uint64_t)m->ny, (uint64_t)m->nz, (uint64_t)m->p,
                           (uint64_t)m->q};
  if (fwrite(hdr, sizeof(uint64_t), 6, fp.f) != 6) return DGB_ERR_IO;
  const int64_t b6[6] = {m->bounds[0], m->bounds[1], m->bounds[2], m->bounds[3], m->bounds[4], m->bounds[5]};
  if (fwrite(b6, sizeof(int64_t), 6, fp.f) != 6) return DGB_ERR_IO;
  const uint64_t nout = order.size();
  if (fwrite(&nout, sizeof nout, 1, fp.f) != 1) return DGB_ERR_IO;
  if (fwrite(m->nodes, sizeof(double), E * nq * 3, fp.f) != E * nq * 3) return DGB_ERR_IO;
  for (int k : order) {
    const uint64_t kl = strlen(keys[k]);
    if (fwrite(&kl, sizeof kl, 1, fp.f) != 1) return DGB_ERR_IO;
    if (kl && fwrite(keys[k], 1, kl, fp.f) != kl) return DGB_ERR_IO;
    if (fwrite(data[k], sizeof(double), E * 5 * nb, fp.f) != E * 5 * nb) return DGB_ERR_IO;
  }
  return DGB_OK;
}

extern "C" int dgb_read_state(const char* fname, unsigned long long* tstep, int* nx, int* ny, int* nz,
                              int* p, int* q, long long* bounds, double* nodes, const char* key,
                              double* data)
{
  if (!fname) return DGB_ERR_ARG;
  File fp(fopen(fname, "rb"));
  if (!fp.f) return DGB_ERR_IO;
  uint64_t hdr[6];
  int64_t b6[6];
  uint64_t nout;
  if (fread(hdr, sizeof(uint64_t), 6, fp.f) != 6) return DGB_ERR_IO;
  if (fread(b6, sizeof(int64_t), 6, fp.f) != 6) return DGB_ERR_IO;
  if (fread(&nout, sizeof nout, 1, fp.f) != 1) return DGB_ERR_IO;
  if (hdr[1] == 0 || hdr[2] == 0 || hdr[3] == 0 || hdr[1] > (1u << 20) || hdr[2] > (1u << 20) ||
      hdr[3] > (1u << 20) || hdr[4] > 16 || hdr[5] > 16 || nout > 1024)
    return DGB_ERR_IO;
  if (tstep) *tstep = hdr[0];
  if (nx) *nx = (int)hdr[1];
  if (ny) *ny = (int)hdr[2];
  if (nz) *nz = (int)hdr[3];
  if (p) *p = (int)hdr[4];
  if (q) *q = (int)hdr[5];
  if (bounds)
    for (int i = 0; i < 6; ++i) bounds[i] = b6[i];
  const uint64_t E = hdr[1] * hdr[2] * hdr[3];
  const uint64_t nq = (hdr[5] + 1) * (hdr[5] + 1) * (hdr[5] + 1);
  const uint64_t nb = (hdr[4] + 1) * (hdr[4] + 1) * (hdr[4] + 1);
  std::vector<double> buf;
  if (nodes) {
    if (fread(nodes, sizeof(double), E * nq * 3, fp.f) != E * nq * 3) return DGB_ERR_IO;
  } else if (fseek(fp.f, (long)(E * nq * 3 * sizeof(double)), SEEK_CUR) != 0) {
    return DGB_ERR_IO;
  }
  bool found = key == nullptr;
  for (uint64_t o = 0; o < nout; ++o) {
    uint64_t kl;
    if (fread(&kl, sizeof kl, 1, fp.f) != 1 || kl > 1023) return DGB_ERR_IO;
    char name[1024];
    if (kl && fread(name, 1, kl, fp.f) != kl) return DGB_ERR_IO;
    name[kl] = '\0';
    const bool match = key && strcmp(name, key) == 0;
    if (match) found = true;
    if (match && data) {
      if (fread(data, sizeof(double), E * 5 * nb, fp.f) != E * 5 * nb) return DGB_ERR_IO;
    } else {
      // skip, but verify the payload is present
      buf.resize(E * 5 * nb);
      if (fread(buf.data(), sizeof(double), E * 5 * nb, fp.f) != E * 5 * nb) return DGB_ERR_IO;
    }
  }
  return found ? DGB_OK : DGB_ERR_IO;
}
