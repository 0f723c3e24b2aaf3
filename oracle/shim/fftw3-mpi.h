// Stand-in for <fftw3-mpi.h> (FFTW 3.3.x, absent from this image) that lets
// the reference's own quasi/quasi.cpp and quasi/quasi-stb.cpp compile and run
// with MPI ranks emulated as threads of one process.
//
// TEST INFRASTRUCTURE ONLY (the oracle's pin).  It declares exactly the
// subset of the FFTW-MPI and MPI-2 C++ APIs those two files call:
//   fftw_mpi_init, fftw_mpi_local_size_3d, fftw_mpi_plan_r2r_3d,
//   fftw_execute, fftw_destroy_plan, fftw_cleanup          (quasi.cpp:229-495,2312-2320)
//   MPI::Init/Finalize, COMM_WORLD.{Get_rank,Get_size,Send,Recv,Reduce,
//   Bcast,Gather,Barrier}                                   (quasi.cpp:228-2323)
// The r2r kinds follow FFTW's published definitions (oracle/shim/r2r_cpu.hpp).
#pragma once
#include <cstddef>
#include "quasi_mpi_shim.h"

typedef int fftw_r2r_kind;
enum { FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
       FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
       FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10 };
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

struct quasi_shim_plan;
typedef quasi_shim_plan* fftw_plan;

void fftw_mpi_init();
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, const MPI::Intracomm& comm,
                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start);
fftw_plan fftw_mpi_plan_r2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, double* out,
                               const MPI::Intracomm& comm, fftw_r2r_kind kind0, fftw_r2r_kind kind1,
                               fftw_r2r_kind kind2, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
void fftw_cleanup();

// Run-time knobs the build recipe substitutes into its patched copy of the
// reference (grid size, output prefix, step cap, dump cadence).
long quasi_shim_grid(int axis);
const char* quasi_shim_outdir();
int quasi_shim_int(const char* name, int dflt);
