// dgb: command-line driver over the dgb200 C ABI, a drop-in for the
// reference's GPU driver solver/cudg.cu.  Same options with the same defaults
// (solver_inputs and parse_solver_inputs, input.cpp:23-125, parsed like
// optparse, io.cpp:194-300), the same mesh (the bump channel,
// geometry_common.cpp:494-576, or a .dg input file), the same initial
// conditions (uniform / turbulent, solver_init.cpp:22-77), the same per-step
// residual-norm lines and the same checkpoint and final .dg files
// (cudg.cu:108-143, io.cpp:33-90).  Host code only: all compute runs in the
// library's CUDA kernels.
//
// Differences: the arithmetic is FP64 (or -precision mixed), not the
// reference GPU build's FP32; -npx/-npy/-npz must be 1 (one GPU).  The
// running mean (-mean_start) follows the reference's CPU driver dg.cpp, which
// has it (cudg.cu does not).  -prandtl adds the optional heat flux (an
// extension; 0, the default, is the reference's physics).
#include <cuda_runtime.h>

#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dgb200.h"

namespace {

struct Inputs {
  unsigned long long p = 1, q = 2;
  unsigned long long nx = 6, ny = 4, nz = 4;
  double lx = 2., ly = 1., lz = 1.;
  unsigned long long npx = 1, npy = 1, npz = 1;
  double stretch = 0., bmp_h = 0.1, bmp_c = 1.0, bmp_v = 0.05;
  long long bnd[6] = {DGB_BT_SUBSONIC_INFLOW, DGB_BT_SUBSONIC_OUTFLOW, DGB_BT_INVISCID_WALL,
                      DGB_BT_INVISCID_WALL,   DGB_BT_PERIODIC,         DGB_BT_PERIODIC};
  double gamma = 1.4, gcnst = 287., mu = 1e-3, c = 1.0, rho = 1.0, u = 0.1, v = 0., w = 0.;
  std::string ofile = "output", ifile;
  double dt = 1e-4;
  unsigned long long niter = 1000, chkint = 1000, mean_start = 1ULL << 63;
  int scheme = DGB_TVDRK3;
  double eta = 6.;
  double source[5] = {0., 0., 0., 0., 0.};
  bool turb = false;
  int precision = DGB_FP64;
  double prandtl = 0.;
  double twall = -1.;  // isothermal walls' temperature (< 0: the reference temperature)
  bool timing = false;  // report the stepping loop's wall time on stderr
  bool chksync = false;  // write each checkpoint before the next step, as cudg.cu does
};

enum Kind { K_U64, K_DBL, K_STR, K_BOOL, K_BTYPE, K_SCHEME, K_PREC };

struct Opt {
  const char* name;
  const char* help;
  Kind kind;
  void* data;
};

bool btype_of(const char* s, long long* out)
{
  // the reference's boundary_types map (boundaries.cpp:37-44)
  static const struct {
    const char* n;
    long long v;
  } map[] = {{"periodic", DGB_BT_PERIODIC},
             {"freestream", DGB_BT_FREESTREAM},
             {"inviscid_wall", DGB_BT_INVISCID_WALL},
             {"subsonic_inflow", DGB_BT_SUBSONIC_INFLOW},
             {"subsonic_outflow", DGB_BT_SUBSONIC_OUTFLOW},
             {"no_slip_wall", DGB_BT_NO_SLIP_WALL},
             {"isothermal_wall", DGB_BT_ISOTHERMAL_WALL}};  // an extension (-twall)
  for (const auto& m : map)
    if (!strcmp(s, m.n)) {
      *out = m.v;
      return true;
    }
  return false;
}

// returns 1 after printing the option list for -h, 0 otherwise; unknown
// options and values are reported and skipped as the reference does
int parse(int argc, char** argv, Inputs& in)
{
  Opt opts[] = {
      {"p", "solution order", K_U64, &in.p},
      {"q", "geometry order", K_U64, &in.q},
      {"dt", "time step", K_DBL, &in.dt},
      {"niter", "iteration count", K_U64, &in.niter},
      {"chkint", "checkpoint interval", K_U64, &in.chkint},
      {"scheme", "time stepping scheme (RK4, tvdRK3)", K_SCHEME, &in.scheme},
      {"eta", "BR2 stabilization parameter", K_DBL, &in.eta},
      {"turb", "initialize turbulent instead of uniform", K_BOOL, &in.turb},
      {"mean_start", "iteration at which to start averaging", K_U64, &in.mean_start},
      {"gamma", "ratio of specific heats", K_DBL, &in.gamma},
      {"mu", "dynamic viscosity", K_DBL, &in.mu},
      {"c", "speed of sound", K_DBL, &in.c},
      {"rho", "reference density", K_DBL, &in.rho},
      {"u", "reference x velocity", K_DBL, &in.u},
      {"v", "reference y velocity", K_DBL, &in.v},
      {"w", "reference z velocity", K_DBL, &in.w},
      {"fx", "force per unit volume in x", K_DBL, &in.source[1]},
      {"nx", "num elems in x", K_U64, &in.nx},
      {"ny", "num elems in y", K_U64, &in.ny},
      {"nz", "num elems in z", K_U64, &in.nz},
      {"lx", "domain length in x", K_DBL, &in.lx},
      {"ly", "domain length in y", K_DBL, &in.ly},
      {"lz", "domain length in z", K_DBL, &in.lz},
      {"a", "wall normal stretching parameter (0, 1)", K_DBL, &in.stretch},
      {"bmx", "-x boundary type", K_BTYPE, &in.bnd[0]},
      {"bpx", "+x boundary type", K_BTYPE, &in.bnd[1]},
      {"bmy", "-y boundary type", K_BTYPE, &in.bnd[2]},
      {"bpy", "+y boundary type", K_BTYPE, &in.bnd[3]},
      {"bmz", "-z boundary type", K_BTYPE, &in.bnd[4]},
      {"bpz", "+z boundary type", K_BTYPE, &in.bnd[5]},
      {"bmp_h", "bump height", K_DBL, &in.bmp_h},
      {"bmp_c", "bump center in x", K_DBL, &in.bmp_c},
      {"bmp_v", "bump variance", K_DBL, &in.bmp_v},
      {"npx", "processor count in x (1: one GPU)", K_U64, &in.npx},
      {"npy", "processor count in y (1: one GPU)", K_U64, &in.npy},
      {"npz", "processor count in z (1: one GPU)", K_U64, &in.npz},
      {"ofile", "output file prefix", K_STR, &in.ofile},
      {"ifile", "input file prefix", K_STR, &in.ifile},
      {"precision", "arithmetic: fp64 or mixed", K_PREC, &in.precision},
      {"prandtl", "Prandtl number of the heat flux (0: none)", K_DBL, &in.prandtl},
      {"twall", "temperature of isothermal_wall sides (default: reference T)", K_DBL, &in.twall},
      {"timing", "print the stepping loop's wall time (checkpoints included) on stderr", K_BOOL, &in.timing},
      {"chksync", "write each checkpoint before the next step (the reference's order)", K_BOOL, &in.chksync},
  };
  const int nopt = (int)(sizeof opts / sizeof opts[0]);
  if (argc > 1 && !strcmp(argv[1], "-h")) {
    printf("Options:\n");
    for (const Opt& o : opts) printf("  %10s: %s\n", o.name, o.help);
    return 1;
  }
  int head = 1;
  while (head < argc) {
    if (argv[head][0] != '-') {
      printf("ignoring non-option argument %s\n", argv[head]);
      ++head;
      continue;
    }
    int oi = 0;
    for (; oi < nopt; ++oi)
      if (!strcmp(opts[oi].name, argv[head] + 1)) break;
    if (oi == nopt) {
      printf("failed to find option number %d : %s\n", head, argv[head] + 1);
      ++head;
      continue;
    }
    const Opt& o = opts[oi];
    if (o.kind == K_BOOL) {
      *(bool*)o.data = true;
      ++head;
      continue;
    }
    if (head + 1 >= argc) {
      printf("no argument provided for \"%s\" at end of argument list\n", argv[head] + 1);
      ++head;
      continue;
    }
    const char* val = argv[head + 1];
    switch (o.kind) {
      case K_U64: *(unsigned long long*)o.data = strtoull(val, nullptr, 10); break;
      case K_DBL: *(double*)o.data = strtod(val, nullptr); break;
      case K_STR: *(std::string*)o.data = val; break;
      case K_BTYPE:
        if (!btype_of(val, (long long*)o.data)) printf("unknown boundary type \"%s\"\n", val);
        break;
      case K_SCHEME:  // multistage_schemes (time.cpp:29-31)
        if (!strcmp(val, "RK4"))
          *(int*)o.data = DGB_RK4;
        else if (!strcmp(val, "tvdRK3"))
          *(int*)o.data = DGB_TVDRK3;
        else
          printf("unknown time scheme \"%s\"\n", val);
        break;
      case K_PREC:
        if (!strcmp(val, "fp64"))
          *(int*)o.data = DGB_FP64;
        else if (!strcmp(val, "mixed"))
          *(int*)o.data = DGB_MIXED_FP32;
        else
          printf("unknown precision \"%s\"\n", val);
        break;
      case K_BOOL: break;
    }
    head += 2;
  }
  return 0;
}

[[noreturn]] void die(const char* what, int rc)
{
  fprintf(stderr, "dgb: %s: %s (%s)\n", what, dgb_error_string(rc), dgb_last_error_message());
  exit(1);
}

// physical position of the order-p solution node b of element e through the
// order-q isoparametric map (ref2glo at lagrange_node3d, basis.cpp:79-85)
void node_position(const double* X, int p, int q, int b, double* x)
{
  const int P = p + 1, Q = q + 1;
  const int ix = b % P, iy = (b / P) % P, iz = b / (P * P);
  const double r[3] = {p ? (double)ix / p : 0., p ? (double)iy / p : 0., p ? (double)iz / p : 0.};
  x[0] = x[1] = x[2] = 0.;
  for (int k = 0; k < Q; ++k)
    for (int j = 0; j < Q; ++j)
      for (int i = 0; i < Q; ++i) {
        const double phi = dgb_lagrange1d(i, q, r[0]) * dgb_lagrange1d(j, q, r[1]) * dgb_lagrange1d(k, q, r[2]);
        const double* n = X + 3 * (i + Q * (j + Q * k));
        for (int c = 0; c < 3; ++c) x[c] += n[c] * phi;
      }
}

// turbulent initial state (solver_init.cpp:29-77): four octaves of a
// sine-product velocity perturbation at a tenth of the reference speed
void turbulent(const dgb_params& prm, int p, int q, long E, const double* nodes, double l, double* U)
{
  const double twopi = 2. * M_PI, offst = 0.3;
  const double rho = prm.Ufr[0];
  const double vel0[3] = {prm.Ufr[1] / rho, prm.Ufr[2] / rho, prm.Ufr[3] / rho};
  const double amp = std::sqrt(vel0[0] * vel0[0] + vel0[1] * vel0[1] + vel0[2] * vel0[2]) / 10.;
  const int NB = (p + 1) * (p + 1) * (p + 1), NQ = (q + 1) * (q + 1) * (q + 1);
  for (long e = 0; e < E; ++e)
    for (int b = 0; b < NB; ++b) {
      double g[3];
      node_position(nodes + (size_t)e * NQ * 3, p, q, b, g);
      double vel[3] = {vel0[0], vel0[1], vel0[2]};
      for (int i = 0; i < 3; ++i)
        for (double f : {0.5, 0.25, 0.125, 0.0625})
          vel[i] += amp * (std::sin(twopi * ((g[0] - i * offst) / (f * l))) *
                           std::sin(twopi * ((g[1] - i * offst) / (f * l))) *
                           std::sin(twopi * ((g[2] - i * offst) / (f * l))));
      double* u = U + (size_t)e * 5 * NB;
      u[b] = prm.Ufr[0];
      u[NB + b] = vel[0] * rho;
      u[2 * NB + b] = vel[1] * rho;
      u[3 * NB + b] = vel[2] * rho;
      u[4 * NB + b] = prm.Ufr[4];
    }
}

}  // namespace

int main(int argc, char** argv)
{
  Inputs in;
  if (parse(argc, argv, in)) return 0;
  if (in.npx != 1 || in.npy != 1 || in.npz != 1) {
    fprintf(stderr, "dgb: one GPU, one domain: -npx/-npy/-npz must be 1\n");
    return 1;
  }
  dgb_params prm;
  int rc = dgb_make_reference_state(in.gamma, in.gcnst, in.mu, in.c, in.rho, in.u, in.v, in.w, in.eta, in.source,
                                    &prm);
  if (rc) die("reference state", rc);

  unsigned long long tstep = 0;
  dgb_mesh_desc mesh;
  std::vector<double> nodes, U;
  if (in.ifile.empty()) {
    mesh.nx = (int)in.nx;
    mesh.ny = (int)in.ny;
    mesh.nz = (int)in.nz;
    mesh.p = (int)in.p;
    mesh.q = (int)in.q;
    for (int s = 0; s < 6; ++s) mesh.bounds[s] = in.bnd[s];
    const long E = (long)in.nx * in.ny * in.nz;
    nodes.resize((size_t)E * (in.q + 1) * (in.q + 1) * (in.q + 1) * 3);
    rc = dgb_bump_nodes(mesh.nx, mesh.ny, mesh.nz, mesh.q, in.lx, in.ly, in.lz, in.stretch, in.bmp_h, in.bmp_c,
                        in.bmp_v, nodes.data());
    if (rc) die("mesh", rc);
    const int NB = (mesh.p + 1) * (mesh.p + 1) * (mesh.p + 1);
    U.resize((size_t)E * 5 * NB);
    if (in.turb) {
      turbulent(prm, mesh.p, mesh.q, E, nodes.data(), in.lx, U.data());
    } else {  // uniform (solver_init.cpp:21-27)
      for (long e = 0; e < E; ++e)
        for (int r = 0; r < 5; ++r)
          for (int b = 0; b < NB; ++b) U[((size_t)e * 5 + r) * NB + b] = prm.Ufr[r];
    }
  } else {
    const std::string f = in.ifile + ".dg";
    int nx, ny, nz, p, q;
    long long bounds[6];
    rc = dgb_read_state(f.c_str(), &tstep, &nx, &ny, &nz, &p, &q, bounds, nullptr, "state", nullptr);
    if (rc) die(f.c_str(), rc);
    const long E = (long)nx * ny * nz;
    nodes.resize((size_t)E * (q + 1) * (q + 1) * (q + 1) * 3);
    U.resize((size_t)E * 5 * (p + 1) * (p + 1) * (p + 1));
    rc = dgb_read_state(f.c_str(), &tstep, &nx, &ny, &nz, &p, &q, bounds, nodes.data(), "state", U.data());
    if (rc) die(f.c_str(), rc);
    mesh.nx = nx;
    mesh.ny = ny;
    mesh.nz = nz;
    mesh.p = p;
    mesh.q = q;
    for (int s = 0; s < 6; ++s) mesh.bounds[s] = bounds[s];
    tstep += 1;  // starting on the step after the one that was read (cudg.cu:69)
  }
  mesh.nodes = nodes.data();

  dgb_handle* h = nullptr;
  if ((rc = dgb_create(&mesh, &prm, in.precision, &h))) die("dgb_create", rc);
  if ((rc = dgb_set_prandtl(h, in.prandtl))) die("dgb_set_prandtl", rc);
  if (in.twall > 0. && (rc = dgb_set_wall_temperature(h, in.twall))) die("dgb_set_wall_temperature", rc);
  if ((rc = dgb_set_state(h, U.data()))) die("dgb_set_state", rc);

  // checkpoints are written while the steps go on: the state is copied to
  // a device snapshot (a device-to-device copy on the handle's stream), the
  // snapshot goes to pinned host memory on a copy stream, and a host thread
  // writes the .dg file once that copy is done.  The next checkpoint waits
  // for the previous file before it reuses the buffers.
  struct Writer {
    cudaStream_t copy = nullptr;
    cudaEvent_t done = nullptr;
    double* d_snap = nullptr;
    double* h_state = nullptr;
    std::thread th;
    int rc = DGB_OK;
    std::string file;
    void wait()
    {
      if (th.joinable()) th.join();
      if (rc) die(file.c_str(), rc);
    }
    ~Writer()
    {
      if (th.joinable()) th.join();
      if (d_snap) cudaFree(d_snap);
      if (h_state) cudaFreeHost(h_state);
      if (done) cudaEventDestroy(done);
      if (copy) cudaStreamDestroy(copy);
    }
  } writer;
  auto cuda_ok = [](cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
      fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
      exit(1);
    }
  };
  auto writer_buffers = [&]() {  // made at the first checkpoint (whichever step index it falls on)
    if (writer.d_snap) return;
    const size_t bytes = sizeof(double) * U.size();
    cuda_ok(cudaStreamCreateWithFlags(&writer.copy, cudaStreamNonBlocking), "checkpoint stream");
    cuda_ok(cudaEventCreateWithFlags(&writer.done, cudaEventDisableTiming), "checkpoint event");
    cuda_ok(cudaMalloc(&writer.d_snap, bytes), "checkpoint snapshot");
    cuda_ok(cudaMallocHost(&writer.h_state, bytes), "checkpoint host buffer");
  };

  // running mean (dg.cpp:123-131): an input file may carry one to continue
  std::vector<double> M(U.size());
  bool have_mean = false;
  if (!in.ifile.empty()) {
    const std::string f = in.ifile + ".dg";
    if (dgb_read_state(f.c_str(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, "mean",
                       M.data()) == DGB_OK) {
      if ((rc = dgb_set_mean(h, M.data()))) die("dgb_set_mean", rc);
      have_mean = true;
    }
  }

  const char* keys[2] = {"state", "mean"};
  const double* data[2] = {U.data(), M.data()};
  auto write = [&](const std::string& f, unsigned long long ts) {
    int r = dgb_get_state(h, U.data());
    if (r) die("dgb_get_state", r);
    if (have_mean && (r = dgb_get_mean(h, M.data()))) die("dgb_get_mean", r);
    r = dgb_write_state(f.c_str(), ts, &mesh, have_mean ? 2 : 1, keys, data);
    if (r) die(f.c_str(), r);
  };

  // time stepping: the reference checkpoints before the step whose index
  // satisfies (tstep + 1) % chkint == 0 (cudg.cu:112-130); between checkpoints
  // the steps run as one dgb_step call (one CUDA graph replay per step), or
  // one at a time once the running mean is being accumulated
  const unsigned long long tfinal = tstep + in.niter, tstart = tstep;
  const auto t_loop = std::chrono::steady_clock::now();
  std::vector<double> norms;
  while (tstep < tfinal) {
    if (in.chkint && (tstep + 1) % in.chkint == 0) {
      char f[1100];
      snprintf(f, sizeof f, "%s%" PRIu64 ".dg", in.ofile.c_str(), (uint64_t)tstep);
      writer.wait();  // the previous checkpoint's file is written: its buffers are free
      writer_buffers();
      if ((rc = dgb_get_state_device(h, writer.d_snap))) die("dgb_get_state_device", rc);
      // continue from the state as written, as a restart from this file
      // would (dgb_step otherwise continues from its Gauss-point copy)
      if ((rc = dgb_set_state_device(h, writer.d_snap))) die("dgb_set_state_device", rc);
      const bool with_mean = have_mean;
      if (with_mean && (rc = dgb_get_mean(h, M.data()))) die("dgb_get_mean", rc);
      cuda_ok(cudaMemcpyAsync(writer.h_state, writer.d_snap, sizeof(double) * U.size(), cudaMemcpyDeviceToHost,
                              writer.copy),
              "checkpoint copy");
      cuda_ok(cudaEventRecord(writer.done, writer.copy), "checkpoint event");
      writer.file = f;
      writer.rc = DGB_OK;
      writer.th = std::thread([&writer, &mesh, &M, with_mean, ts = tstep, file = std::string(f)]() {
        if (cudaEventSynchronize(writer.done) != cudaSuccess) {
          writer.rc = DGB_ERR_CUDA;
          return;
        }
        const char* k[2] = {"state", "mean"};
        const double* d[2] = {writer.h_state, M.data()};
        writer.rc = dgb_write_state(file.c_str(), ts, &mesh, with_mean ? 2 : 1, k, d);
      });
      if (with_mean || in.chksync) writer.wait();  // the mean's host copy is reused by the next update
    }
    unsigned long long n = tfinal - tstep;
    if (in.chkint) {  // up to, not including, the next checkpointing step
      const unsigned long long next = ((tstep + 1) / in.chkint + 1) * in.chkint - 1;
      if (next > tstep && next - tstep < n) n = next - tstep;
      if (n == 0) n = 1;
    }
    if (tstep >= in.mean_start)
      n = 1;
    else if (in.mean_start - tstep < n)
      n = in.mean_start - tstep;
    norms.resize(n);
    rc = dgb_step(h, in.scheme, in.dt, n, norms.data());
    if (rc == DGB_OK || rc == DGB_ERR_NONFINITE) {  // the reference prints up to the NaN, then aborts
      for (unsigned long long k = 0; k < n; ++k) {
        printf("%" PRIu64 " : %.17e\n", (uint64_t)(tstep + k), norms[k]);
        if (!std::isfinite(norms[k])) break;
      }
    }
    if (rc) die("dgb_step", rc);
    tstep += n;
    if (tstep - 1 >= in.mean_start) {  // after step tstep - 1 (n == 1 here)
      if ((rc = dgb_mean_update(h, tstep - 1, in.mean_start))) die("dgb_mean_update", rc);
      have_mean = true;
    }
  }
  writer.wait();
  if (in.timing) {  // the steps and every checkpoint file, not the set-up or the final file
    const double s_loop = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count();
    fprintf(stderr, "dgb: %" PRIu64 " steps in %.6f s (%.6f ms/step)\n", (uint64_t)(tstep - tstart), s_loop,
            tstep > tstart ? 1e3 * s_loop / (double)(tstep - tstart) : 0.);
  }
  write(in.ofile + ".dg", tstep - 1);  // the index of the last step taken, as cudg.cu:140-141 writes
  dgb_destroy(h);
  return 0;
}
