/*
 * mpi.h -- a small multi-process stand-in for MPI, enough to compile and run
 * the reference's particle path (LATfield2_parallel2d*.hpp, Lattice, Field,
 * Particles) where no MPI is installed.  TEST INFRASTRUCTURE ONLY: it builds
 * the reference-compiled checker under oracle/_ref.
 *
 * Model: MPI_Init forks LF2_MINIMPI_NP - 1 children (default 1 process = no
 * fork).  Every pair of processes shares a Unix socketpair created before the
 * fork.  Point-to-point messages carry (communicator, tag, length) headers and
 * are matched per source in arrival order, like MPI's non-overtaking rule;
 * messages to self go through an in-process queue.  Collectives run through
 * member 0 of the communicator and reduce in member order.  A receive from
 * self with nothing queued aborts with a message instead of blocking forever
 * (the reference's moveParticles does that on a 1x1 process grid).
 *
 * Header-only: include it in exactly one translation unit.
 */
#ifndef LF2_MINIMPI_H
#define LF2_MINIMPI_H

#include <errno.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/prctl.h>
#include <sys/socket.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <unistd.h>

#include <deque>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_GROUP_NULL (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_FLOAT 4
#define MPI_DOUBLE 5
#define MPI_UNSIGNED 6
#define MPI_LONG_LONG 7
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

namespace lf2_minimpi {

struct Msg {
  int comm, tag;
  std::vector<char> data;
};

struct State {
  int rank = 0, size = 1;
  bool finalized = false;
  std::vector<int> fd;                      // fd[r]: socket to world rank r
  std::vector<std::deque<Msg>> pending;     // pending[r]: unmatched messages from r
  std::vector<std::vector<int>> comms;      // members (world ranks) of each communicator
  std::vector<std::vector<int>> groups;     // members (world ranks) of each group
  std::vector<pid_t> children;
};

inline State& st()
{
  static State s;
  return s;
}

inline void die(const char* what)
{
  fprintf(stderr, "minimpi rank %d: %s\n", st().rank, what);
  fflush(stderr);
  kill(0, SIGKILL);  // the whole job (its own process group, see MPI_Init)
  _exit(70);
}

inline bool tracing()
{
  static const bool t = getenv("LF2_MINIMPI_TRACE") != nullptr;
  return t;
}

inline void write_all(int fd, const void* p, size_t n)
{
  const char* c = (const char*)p;
  while (n) {
    ssize_t w = ::write(fd, c, n);
    if (w < 0) {
      if (errno == EINTR) continue;
      die("socket write failed");
    }
    c += w;
    n -= (size_t)w;
  }
}

inline void read_all(int fd, void* p, size_t n)
{
  char* c = (char*)p;
  while (n) {
    ssize_t r = ::read(fd, c, n);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) die("peer closed its socket");
    c += r;
    n -= (size_t)r;
  }
}

inline int world_of(MPI_Comm comm, int r)
{
  if (comm < 0 || comm >= (int)st().comms.size()) die("bad communicator");
  const std::vector<int>& m = st().comms[comm];
  if (r < 0 || r >= (int)m.size()) die("rank outside communicator");
  return m[r];
}

inline int my_index(const std::vector<int>& m)
{
  for (size_t i = 0; i < m.size(); i++)
    if (m[i] == st().rank) return (int)i;
  return MPI_UNDEFINED;
}

inline void send_raw(int dest_world, int comm, int tag, const void* buf, size_t len)
{
  State& s = st();
  if (tracing()) fprintf(stderr, "[%d] send -> %d comm %d tag %d len %zu\n", s.rank, dest_world, comm, tag, len);
  if (dest_world == s.rank) {
    Msg m;
    m.comm = comm;
    m.tag = tag;
    m.data.assign((const char*)buf, (const char*)buf + len);
    s.pending[s.rank].push_back(m);
    return;
  }
  long long hdr[3] = {comm, tag, (long long)len};
  write_all(s.fd[dest_world], hdr, sizeof hdr);
  if (len) write_all(s.fd[dest_world], buf, len);
}

inline size_t recv_raw(int src_world, int comm, int tag, void* buf, size_t cap)
{
  State& s = st();
  if (tracing()) fprintf(stderr, "[%d] recv <- %d comm %d tag %d cap %zu\n", s.rank, src_world, comm, tag, cap);
  std::deque<Msg>& q = s.pending[src_world];
  for (;;) {
    for (auto it = q.begin(); it != q.end(); ++it) {
      if (it->comm == comm && it->tag == tag) {
        const size_t n = it->data.size();
        if (n > cap) die("message longer than the receive buffer");
        if (n) memcpy(buf, it->data.data(), n);
        q.erase(it);
        return n;
      }
    }
    if (src_world == s.rank) die("receive from self with no message queued (would deadlock)");
    long long hdr[3];
    read_all(s.fd[src_world], hdr, sizeof hdr);
    Msg m;
    m.comm = (int)hdr[0];
    m.tag = (int)hdr[1];
    m.data.resize((size_t)hdr[2]);
    if (hdr[2]) read_all(s.fd[src_world], m.data.data(), (size_t)hdr[2]);
    q.push_back(m);
  }
}

inline size_t type_size(MPI_Datatype t)
{
  switch (t) {
    case MPI_BYTE: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_UNSIGNED: return sizeof(unsigned);
    case MPI_LONG_LONG: return sizeof(long long);
  }
  die("unsupported datatype");
  return 0;
}

template <typename T>
inline void reduce_into(T* acc, const T* in, int n, MPI_Op op)
{
  for (int i = 0; i < n; i++) {
    if (op == MPI_SUM) acc[i] += in[i];
    else if (op == MPI_MIN) acc[i] = in[i] < acc[i] ? in[i] : acc[i];
    else if (op == MPI_MAX) acc[i] = in[i] > acc[i] ? in[i] : acc[i];
    else die("unsupported op");
  }
}

inline void reduce_typed(void* acc, const void* in, int n, MPI_Datatype t, MPI_Op op)
{
  switch (t) {
    case MPI_BYTE: reduce_into((unsigned char*)acc, (const unsigned char*)in, n, op); break;
    case MPI_INT: reduce_into((int*)acc, (const int*)in, n, op); break;
    case MPI_LONG: reduce_into((long*)acc, (const long*)in, n, op); break;
    case MPI_FLOAT: reduce_into((float*)acc, (const float*)in, n, op); break;
    case MPI_DOUBLE: reduce_into((double*)acc, (const double*)in, n, op); break;
    case MPI_UNSIGNED: reduce_into((unsigned*)acc, (const unsigned*)in, n, op); break;
    case MPI_LONG_LONG: reduce_into((long long*)acc, (const long long*)in, n, op); break;
    default: die("unsupported reduction datatype");
  }
}

const int TAG_COLL = -1000;

// Data to the communicator's member 0, which combines in member order.
inline void coll_reduce_to_root(MPI_Comm comm, void* data, size_t bytes, int count, MPI_Datatype t,
                                MPI_Op op)
{
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  if (me == 0) {
    std::vector<char> tmp(bytes);
    for (size_t i = 1; i < m.size(); i++) {
      recv_raw(m[i], comm, TAG_COLL, tmp.data(), bytes);
      reduce_typed(data, tmp.data(), count, t, op);
    }
  } else {
    send_raw(m[0], comm, TAG_COLL, data, bytes);
  }
}

inline void coll_bcast_from(MPI_Comm comm, int root, void* data, size_t bytes)
{
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  if (me == root) {
    for (size_t i = 0; i < m.size(); i++)
      if ((int)i != root) send_raw(m[i], comm, TAG_COLL - 1, data, bytes);
  } else {
    recv_raw(m[root], comm, TAG_COLL - 1, data, bytes);
  }
}

}  // namespace lf2_minimpi

inline int MPI_Init(int*, char***)
{
  using namespace lf2_minimpi;
  State& s = st();
  const char* e = getenv("LF2_MINIMPI_NP");
  s.size = e ? atoi(e) : 1;
  if (s.size < 1 || s.size > 64) die("LF2_MINIMPI_NP must be 1..64");
  std::vector<std::vector<int>> pair(s.size, std::vector<int>(s.size, -1));
  for (int i = 0; i < s.size; i++)
    for (int j = i + 1; j < s.size; j++) {
      int sv[2];
      if (socketpair(AF_UNIX, SOCK_STREAM, 0, sv) != 0) die("socketpair failed");
      int big = 8 << 20;
      setsockopt(sv[0], SOL_SOCKET, SO_SNDBUF, &big, sizeof big);
      setsockopt(sv[1], SOL_SOCKET, SO_SNDBUF, &big, sizeof big);
      pair[i][j] = sv[0];
      pair[j][i] = sv[1];
    }
  s.rank = 0;
  setpgid(0, 0);  // MPI_Abort signals this job's process group only
  fflush(stdout);
  fflush(stderr);
  for (int r = 1; r < s.size; r++) {
    pid_t p = fork();
    if (p < 0) die("fork failed");
    if (p == 0) {
      s.rank = r;
      s.children.clear();
      prctl(PR_SET_PDEATHSIG, SIGKILL);  // never outlive rank 0
      if (getppid() == 1) _exit(72);
      break;
    }
    s.children.push_back(p);
  }
  s.fd.assign(s.size, -1);
  for (int i = 0; i < s.size; i++)
    for (int j = 0; j < s.size; j++)
      if (i != j) {
        if (i == s.rank) s.fd[j] = pair[i][j];
        else if (j != s.rank) close(pair[i][j]);
      }
  s.pending.assign(s.size, std::deque<Msg>());
  std::vector<int> all;
  for (int r = 0; r < s.size; r++) all.push_back(r);
  s.comms.assign(1, all);
  return MPI_SUCCESS;
}

inline int MPI_Finalized(int* flag)
{
  *flag = lf2_minimpi::st().finalized ? 1 : 0;
  return MPI_SUCCESS;
}

inline int MPI_Finalize()
{
  using namespace lf2_minimpi;
  State& s = st();
  s.finalized = true;
  int bad = 0;
  for (pid_t p : s.children) {
    int status = 0;
    waitpid(p, &status, 0);
    if (!WIFEXITED(status) || WEXITSTATUS(status) != 0) bad = 1;
  }
  if (bad) {
    fprintf(stderr, "minimpi: a child rank failed\n");
    _exit(71);
  }
  return MPI_SUCCESS;
}

inline int MPI_Abort(MPI_Comm, int code)
{
  fprintf(stderr, "minimpi rank %d: MPI_Abort(%d)\n", lf2_minimpi::st().rank, code);
  fflush(stderr);
  kill(0, SIGTERM);
  _exit(code ? code : 1);
}

inline int MPI_Comm_rank(MPI_Comm comm, int* r)
{
  *r = lf2_minimpi::my_index(lf2_minimpi::st().comms[comm]);
  return MPI_SUCCESS;
}

inline int MPI_Comm_size(MPI_Comm comm, int* n)
{
  *n = (int)lf2_minimpi::st().comms[comm].size();
  return MPI_SUCCESS;
}

inline int MPI_Comm_group(MPI_Comm comm, MPI_Group* g)
{
  lf2_minimpi::State& s = lf2_minimpi::st();
  s.groups.push_back(s.comms[comm]);
  *g = (int)s.groups.size() - 1;
  return MPI_SUCCESS;
}

inline int MPI_Group_range_incl(MPI_Group g, int n, int ranges[][3], MPI_Group* out)
{
  lf2_minimpi::State& s = lf2_minimpi::st();
  const std::vector<int> src = s.groups[g];
  std::vector<int> m;
  for (int k = 0; k < n; k++) {
    const int first = ranges[k][0], last = ranges[k][1], stride = ranges[k][2];
    if (stride == 0) lf2_minimpi::die("zero stride");
    for (int r = first; stride > 0 ? r <= last : r >= last; r += stride) m.push_back(src[r]);
  }
  s.groups.push_back(m);
  *out = (int)s.groups.size() - 1;
  return MPI_SUCCESS;
}

inline int MPI_Group_rank(MPI_Group g, int* r)
{
  *r = lf2_minimpi::my_index(lf2_minimpi::st().groups[g]);
  return MPI_SUCCESS;
}

inline int MPI_Group_free(MPI_Group* g)
{
  *g = MPI_GROUP_NULL;
  return MPI_SUCCESS;
}

// Collective over `comm`: every process creates the communicator id in the
// same order, members get it, the others get MPI_COMM_NULL.
inline int MPI_Comm_create(MPI_Comm, MPI_Group g, MPI_Comm* out)
{
  lf2_minimpi::State& s = lf2_minimpi::st();
  s.comms.push_back(s.groups[g]);
  const int id = (int)s.comms.size() - 1;
  *out = lf2_minimpi::my_index(s.groups[g]) == MPI_UNDEFINED ? MPI_COMM_NULL : id;
  return MPI_SUCCESS;
}

inline int MPI_Comm_free(MPI_Comm* c)
{
  *c = MPI_COMM_NULL;
  return MPI_SUCCESS;
}

inline int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  send_raw(world_of(comm, dest), comm, tag, buf, (size_t)count * type_size(t));
  return MPI_SUCCESS;
}

inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm,
                    MPI_Status* status)
{
  using namespace lf2_minimpi;
  recv_raw(world_of(comm, src), comm, tag, buf, (size_t)count * type_size(t));
  if (status) {
    status->MPI_SOURCE = src;
    status->MPI_TAG = tag;
    status->MPI_ERROR = 0;
  }
  return MPI_SUCCESS;
}

inline int MPI_Barrier(MPI_Comm comm)
{
  using namespace lf2_minimpi;
  if (comm == MPI_COMM_NULL) return MPI_SUCCESS;
  char c = 0;
  coll_reduce_to_root(comm, &c, 1, 1, MPI_BYTE, MPI_SUM);
  coll_bcast_from(comm, 0, &c, 1);
  return MPI_SUCCESS;
}

inline int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  if (comm == MPI_COMM_NULL) return MPI_SUCCESS;
  coll_bcast_from(comm, root, buf, (size_t)count * type_size(t));
  return MPI_SUCCESS;
}

inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op,
                         MPI_Comm comm)
{
  using namespace lf2_minimpi;
  const size_t bytes = (size_t)count * type_size(t);
  if (sendbuf != MPI_IN_PLACE && sendbuf != recvbuf) memcpy(recvbuf, sendbuf, bytes);
  coll_reduce_to_root(comm, recvbuf, bytes, count, t, op);
  coll_bcast_from(comm, 0, recvbuf, bytes);
  return MPI_SUCCESS;
}

inline int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op,
                      int root, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  const size_t bytes = (size_t)count * type_size(t);
  std::vector<char> tmp(bytes);
  memcpy(tmp.data(), sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf, bytes);
  coll_reduce_to_root(comm, tmp.data(), bytes, count, t, op);
  // member 0 holds the result; hand it to the root
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  if (root == 0) {
    if (me == 0) memcpy(recvbuf, tmp.data(), bytes);
  } else if (me == 0) {
    send_raw(m[root], comm, TAG_COLL - 2, tmp.data(), bytes);
  } else if (me == root) {
    recv_raw(m[0], comm, TAG_COLL - 2, recvbuf, bytes);
  }
  return MPI_SUCCESS;
}

inline int MPI_Gather(const void* sendbuf, int scount, MPI_Datatype st_, void* recvbuf, int rcount,
                      MPI_Datatype rt, int root, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  const size_t sbytes = (size_t)scount * type_size(st_);
  const size_t rbytes = (size_t)rcount * type_size(rt);
  if (me == root) {
    for (size_t i = 0; i < m.size(); i++) {
      char* dst = (char*)recvbuf + i * rbytes;
      if ((int)i == root) memcpy(dst, sendbuf, sbytes);
      else recv_raw(m[i], comm, TAG_COLL - 3, dst, rbytes);
    }
  } else {
    send_raw(m[root], comm, TAG_COLL - 3, sendbuf, sbytes);
  }
  return MPI_SUCCESS;
}

// Root hands block i of sendbuf to member i.
inline int MPI_Scatter(const void* sendbuf, int scount, MPI_Datatype st_, void* recvbuf, int rcount,
                       MPI_Datatype rt, int root, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  const size_t sbytes = (size_t)scount * type_size(st_);
  const size_t rbytes = (size_t)rcount * type_size(rt);
  if (me == root) {
    for (size_t i = 0; i < m.size(); i++) {
      const char* src = (const char*)sendbuf + i * sbytes;
      if ((int)i == root) memcpy(recvbuf, src, rbytes);
      else send_raw(m[i], comm, TAG_COLL - 4, src, sbytes);
    }
  } else {
    recv_raw(m[root], comm, TAG_COLL - 4, recvbuf, rbytes);
  }
  return MPI_SUCCESS;
}

// Every member sends block j of sendbuf to member j and receives member i's
// block for it into block i of recvbuf.  All sends are queued before the
// receives (the blocks here are small enough for the socket buffers).
inline int MPI_Alltoall(const void* sendbuf, int scount, MPI_Datatype st_, void* recvbuf, int rcount,
                        MPI_Datatype rt, MPI_Comm comm)
{
  using namespace lf2_minimpi;
  const std::vector<int>& m = st().comms[comm];
  const int me = my_index(m);
  const size_t sbytes = (size_t)scount * type_size(st_);
  const size_t rbytes = (size_t)rcount * type_size(rt);
  for (size_t j = 0; j < m.size(); j++)
    if ((int)j != me) send_raw(m[j], comm, TAG_COLL - 5, (const char*)sendbuf + j * sbytes, sbytes);
  memcpy((char*)recvbuf + me * rbytes, (const char*)sendbuf + me * sbytes, rbytes);
  for (size_t i = 0; i < m.size(); i++)
    if ((int)i != me) recv_raw(m[i], comm, TAG_COLL - 5, (char*)recvbuf + i * rbytes, rbytes);
  return MPI_SUCCESS;
}

#endif
