// Implementation of the FFTW-MPI / MPI stand-ins declared in fftw3-mpi.h and
// quasi_mpi_shim.h, plus a process entry point that runs the reference's
// main() once per emulated rank on its own thread.
//
// TEST INFRASTRUCTURE ONLY: it exists so the reference's own translation
// units can produce parity fixtures and a CPU baseline on this machine.
//
// Environment knobs (read once):
//   QUASI_RANKS      emulated MPI rank count (default 2; the reference needs an
//                    even count >= 2, quasi.cpp:1074-1077,1352-1358)
//   QUASI_NX/NY/NZ   grid (default 16 16 32)
//   QUASI_OUTDIR     output prefix; the reference appends "<argv1>-e0d<argv2>/"
//   QUASI_MAXSTEPS   step cap substituted into the time loop
//   QUASI_STEPL1, QUASI_STEPSAVE   diagnostic / dump cadence
//   QUASI_SHIM_THREADS_PER_RANK    unused (one thread per rank)
#include <algorithm>
#include <barrier>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "fftw3-mpi.h"
#include "r2r_cpu.hpp"

void quasi_ref_main(int argc, char* argv[]);

namespace {

int g_size = 2;
thread_local int t_rank = 0;
std::barrier<>* g_barrier = nullptr;

long env_long(const char* name, long dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::strtol(v, nullptr, 10) : dflt;
}

// ---- point to point --------------------------------------------------------
std::mutex g_mail_mu;
std::condition_variable g_mail_cv;
std::map<std::tuple<int, int, int>, std::deque<std::vector<char>>> g_mail;   // (src,dst,tag)

size_t type_size(MPI::Datatype t) { return t == MPI::DOUBLE ? sizeof(double) : sizeof(int); }

// ---- collectives -----------------------------------------------------------
std::vector<const void*> g_slot;

// ---- plans -----------------------------------------------------------------
struct SharedPlan {
  long n0, n1, n2;
  int kind[3];
  std::vector<double*> buf;   // per rank local slab
};
std::mutex g_plan_mu;
std::vector<SharedPlan*> g_plans;
thread_local int t_plan_count = 0;

quasi_cpu::Kind to_kind(int k) {
  switch (k) {
    case FFTW_REDFT10: return quasi_cpu::REDFT10;
    case FFTW_REDFT01: return quasi_cpu::REDFT01;
    case FFTW_RODFT10: return quasi_cpu::RODFT10;
    case FFTW_RODFT01: return quasi_cpu::RODFT01;
    default:
      std::fprintf(stderr, "shim: unsupported r2r kind %d\n", k);
      std::abort();
  }
}

// transform `count` lines of length n starting at base[line_off(l)] with element stride es
template <class LineAddr>
void lines(const quasi_cpu::R2R1D& p, quasi_cpu::Kind kind, long count, long es, LineAddr addr) {
  const long n = p.size();
  std::vector<double> a(n), b(n);
  std::vector<quasi_cpu::cplx> w1, w2;
  for (long l = 0; l < count; l += 2) {
    double* pa = addr(l);
    double* pb = (l + 1 < count) ? addr(l + 1) : nullptr;
    for (long t = 0; t < n; ++t) { a[t] = pa[t * es]; if (pb) b[t] = pb[t * es]; }
    p.pair(kind, a.data(), pb ? b.data() : nullptr, w1, w2);
    for (long t = 0; t < n; ++t) { pa[t * es] = a[t]; if (pb) pb[t * es] = b[t]; }
  }
}

}  // namespace

struct quasi_shim_plan {
  SharedPlan* shared;
};

// ============================================================================
namespace MPI {

Intracomm COMM_WORLD;

void Init() {}
void Finalize() {}

int Intracomm::Get_rank() const { return t_rank; }
int Intracomm::Get_size() const { return g_size; }

void Intracomm::Send(const void* buf, int count, Datatype t, int dest, int tag) const {
  if (dest < 0 || dest >= g_size) {
    std::fprintf(stderr, "shim: rank %d sends to invalid rank %d\n", t_rank, dest);
    std::abort();
  }
  std::vector<char> msg((const char*)buf, (const char*)buf + count * type_size(t));
  {
    std::lock_guard<std::mutex> lk(g_mail_mu);
    g_mail[{t_rank, dest, tag}].push_back(std::move(msg));
  }
  g_mail_cv.notify_all();
}

void Intracomm::Recv(void* buf, int count, Datatype t, int source, int tag) const {
  if (source < 0 || source >= g_size) {
    std::fprintf(stderr, "shim: rank %d receives from invalid rank %d\n", t_rank, source);
    std::abort();
  }
  std::unique_lock<std::mutex> lk(g_mail_mu);
  auto key = std::make_tuple(source, t_rank, tag);
  g_mail_cv.wait(lk, [&] { auto it = g_mail.find(key); return it != g_mail.end() && !it->second.empty(); });
  auto& q = g_mail[key];
  std::vector<char> msg = std::move(q.front());
  q.pop_front();
  size_t bytes = count * type_size(t);
  if (msg.size() != bytes) {
    std::fprintf(stderr, "shim: message size mismatch\n");
    std::abort();
  }
  std::memcpy(buf, msg.data(), bytes);
}

void Intracomm::Barrier() const { g_barrier->arrive_and_wait(); }

void Intracomm::Reduce(const void* sendbuf, void* recvbuf, int count, Datatype t, Op, int root) const {
  g_slot[t_rank] = sendbuf;
  g_barrier->arrive_and_wait();
  if (t_rank == root) {
    for (int c = 0; c < count; ++c) {
      if (t == DOUBLE) {
        double s = 0.0;
        for (int r = 0; r < g_size; ++r) s += ((const double*)g_slot[r])[c];
        ((double*)recvbuf)[c] = s;
      } else {
        int s = 0;
        for (int r = 0; r < g_size; ++r) s += ((const int*)g_slot[r])[c];
        ((int*)recvbuf)[c] = s;
      }
    }
  }
  g_barrier->arrive_and_wait();
}

void Intracomm::Bcast(void* buf, int count, Datatype t, int root) const {
  if (t_rank == root) g_slot[0] = buf;
  g_barrier->arrive_and_wait();
  if (t_rank != root) std::memcpy(buf, g_slot[0], count * type_size(t));
  g_barrier->arrive_and_wait();
}

void Intracomm::Gather(const void* sendbuf, int sendcount, Datatype st, void* recvbuf, int, Datatype,
                       int root) const {
  g_slot[t_rank] = sendbuf;
  g_barrier->arrive_and_wait();
  if (t_rank == root) {
    size_t bytes = sendcount * type_size(st);
    for (int r = 0; r < g_size; ++r) std::memcpy((char*)recvbuf + r * bytes, g_slot[r], bytes);
  }
  g_barrier->arrive_and_wait();
}

}  // namespace MPI

// ============================================================================
long quasi_shim_grid(int axis) {
  static const long n[3] = {env_long("QUASI_NX", 16), env_long("QUASI_NY", 16), env_long("QUASI_NZ", 32)};
  return n[axis];
}

const char* quasi_shim_outdir() {
  const char* v = std::getenv("QUASI_OUTDIR");
  return v ? v : "./quasi_ref_out/run-nu";
}

int quasi_shim_int(const char* name, int dflt) { return (int)env_long(name, dflt); }

void fftw_mpi_init() {}

ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, const MPI::Intracomm&,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
  if (n0 % g_size) {
    std::fprintf(stderr, "shim: Nx=%ld not divisible by %d ranks\n", (long)n0, g_size);
    std::abort();
  }
  *local_n0 = n0 / g_size;
  *local_0_start = t_rank * (n0 / g_size);
  return (n0 / g_size) * n1 * n2;
}

fftw_plan fftw_mpi_plan_r2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, double* out,
                               const MPI::Intracomm&, fftw_r2r_kind k0, fftw_r2r_kind k1, fftw_r2r_kind k2,
                               unsigned) {
  if (in != out) {
    std::fprintf(stderr, "shim: only in-place plans are supported\n");
    std::abort();
  }
  int idx = t_plan_count++;
  SharedPlan* sp;
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if ((int)g_plans.size() <= idx) {
      SharedPlan* p = new SharedPlan{n0, n1, n2, {k0, k1, k2}, std::vector<double*>(g_size, nullptr)};
      g_plans.push_back(p);
    }
    sp = g_plans[idx];
    sp->buf[t_rank] = in;
  }
  g_barrier->arrive_and_wait();
  return new quasi_shim_plan{sp};
}

// Collective execute: every rank transforms y and z on its own slab, then the
// ranks split the (j,k) pencils and transform along x through all slabs.
void fftw_execute(const fftw_plan plan) {
  SharedPlan& sp = *plan->shared;
  const long n0 = sp.n0, n1 = sp.n1, n2 = sp.n2, ln0 = n0 / g_size;
  quasi_cpu::R2R1D px((int)n0), py((int)n1), pz((int)n2);
  g_barrier->arrive_and_wait();
  double* mine = sp.buf[t_rank];
  // z lines (contiguous)
  lines(pz, to_kind(sp.kind[2]), ln0 * n1, 1, [&](long l) { return mine + l * n2; });
  // y lines (stride n2)
  lines(py, to_kind(sp.kind[1]), ln0 * n2, n2, [&](long l) {
    long i = l / n2, k = l % n2;
    return mine + i * n1 * n2 + k;
  });
  g_barrier->arrive_and_wait();
  // x lines: gather each pencil across slabs
  const long total = n1 * n2;
  const long per = (total + g_size - 1) / g_size;
  const long lo = std::min(total, t_rank * per), hi = std::min(total, lo + per);
  std::vector<double> a(n0), b(n0);
  std::vector<quasi_cpu::cplx> w1, w2;
  quasi_cpu::Kind kx = to_kind(sp.kind[0]);
  auto at = [&](long i, long jk) { return sp.buf[i / ln0] + (i % ln0) * total + jk; };
  for (long l = lo; l < hi; l += 2) {
    bool two = l + 1 < hi;
    for (long i = 0; i < n0; ++i) { a[i] = *at(i, l); if (two) b[i] = *at(i, l + 1); }
    px.pair(kx, a.data(), two ? b.data() : nullptr, w1, w2);
    for (long i = 0; i < n0; ++i) { *at(i, l) = a[i]; if (two) *at(i, l + 1) = b[i]; }
  }
  g_barrier->arrive_and_wait();
}

void fftw_destroy_plan(fftw_plan plan) { delete plan; }
void fftw_cleanup() {}

// ============================================================================
int main(int argc, char* argv[]) {
  g_size = (int)env_long("QUASI_RANKS", 2);
  if (g_size < 1) g_size = 1;
  g_slot.assign(g_size, nullptr);
  std::barrier<> bar(g_size);
  g_barrier = &bar;
  std::vector<std::thread> th;
  for (int r = 0; r < g_size; ++r) {
    th.emplace_back([=] {
      t_rank = r;
      quasi_ref_main(argc, argv);
    });
  }
  for (auto& t : th) t.join();
  return 0;
}
