// Minimal MPI-2 C++ binding surface used by quasi.cpp / quasi-stb.cpp, with
// ranks emulated as threads of one process (TEST INFRASTRUCTURE ONLY).
// Point-to-point sends are buffered (never block), which is at least as
// permissive as MPI's eager protocol; collectives are barrier-based and
// deterministic (reductions sum in rank order).
#pragma once

namespace MPI {

enum Datatype { DOUBLE = 1, INT = 2 };
enum Op { SUM = 1 };

class Intracomm {
 public:
  int Get_rank() const;
  int Get_size() const;
  void Send(const void* buf, int count, Datatype t, int dest, int tag) const;
  void Recv(void* buf, int count, Datatype t, int source, int tag) const;
  void Reduce(const void* sendbuf, void* recvbuf, int count, Datatype t, Op op, int root) const;
  void Bcast(void* buf, int count, Datatype t, int root) const;
  void Gather(const void* sendbuf, int sendcount, Datatype st, void* recvbuf, int recvcount,
              Datatype rt, int root) const;
  void Barrier() const;
};

extern Intracomm COMM_WORLD;

void Init();
void Finalize();

}  // namespace MPI
