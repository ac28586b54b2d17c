// Single-process MPI used to build HemePure as the CPU oracle (test infrastructure only).
//
// One rank per communicator.  Datatypes carry a type map (list of byte blocks
// with displacements, a lower bound and an extent) so that derived types built
// with MPI_Type_create_struct — the coalesced point-to-point types of
// net/mixins/pointpoint/CoalescePointPoint.cc and the vector types of
// util/Vector3DHemeLb.cc — pack and unpack exactly as a real MPI would.
// Messages to self are sent eagerly (the payload is packed at send time) and
// matched in posting order by (communicator, tag).
#include "mpi.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

namespace {

struct Block {
  MPI_Aint disp;
  size_t len;
};

struct TypeRec {
  bool live = false;
  size_t size = 0;     // bytes of data per element
  MPI_Aint lb = 0;
  MPI_Aint extent = 0;
  size_t align = 1;
  std::vector<Block> blocks;
};

std::vector<TypeRec>& types() {
  static std::vector<TypeRec> t = [] {
    std::vector<TypeRec> v(17);
    auto prim = [&](int h, size_t s) {
      v[h].live = true;
      v[h].size = s;
      v[h].lb = 0;
      v[h].extent = (MPI_Aint)s;
      v[h].align = s > 16 ? 16 : s;
      v[h].blocks = {{0, s}};
    };
    prim(MPI_CHAR, 1);
    prim(MPI_SIGNED_CHAR, 1);
    prim(MPI_UNSIGNED_CHAR, 1);
    prim(MPI_SHORT, sizeof(short));
    prim(MPI_UNSIGNED_SHORT, sizeof(unsigned short));
    prim(MPI_INT, sizeof(int));
    prim(MPI_UNSIGNED, sizeof(unsigned));
    prim(MPI_LONG, sizeof(long));
    prim(MPI_UNSIGNED_LONG, sizeof(unsigned long));
    prim(MPI_LONG_LONG, sizeof(long long));
    prim(MPI_UNSIGNED_LONG_LONG, sizeof(unsigned long long));
    prim(MPI_FLOAT, sizeof(float));
    prim(MPI_DOUBLE, sizeof(double));
    prim(MPI_LONG_DOUBLE, sizeof(long double));
    prim(MPI_WCHAR, sizeof(wchar_t));
    prim(MPI_BYTE, 1);
    return v;
  }();
  return t;
}

const TypeRec* type_of(MPI_Datatype h) {
  auto& t = types();
  if (h <= 0 || (size_t)h >= t.size() || !t[h].live) return nullptr;
  return &t[h];
}

// Pack `count` elements laid out from `buf` into a contiguous byte string.
bool pack(const void* buf, int count, MPI_Datatype type, std::string& out) {
  const TypeRec* t = type_of(type);
  if (!t || count < 0) return false;
  out.clear();
  out.reserve(t->size * (size_t)count);
  const char* base = (const char*)buf;
  for (int c = 0; c < count; ++c)
    for (const Block& b : t->blocks) out.append(base + c * t->extent + b.disp, b.len);
  return true;
}

// Unpack at most `count` elements; returns the number of bytes consumed.
bool unpack(const std::string& in, void* buf, int count, MPI_Datatype type, size_t* used) {
  const TypeRec* t = type_of(type);
  if (!t || count < 0) return false;
  size_t cap = t->size * (size_t)count;
  if (in.size() > cap) return false;  // truncation
  char* base = (char*)buf;
  size_t pos = 0;
  for (int c = 0; c < count && pos < in.size(); ++c)
    for (const Block& b : t->blocks) {
      if (pos >= in.size()) break;
      size_t n = std::min(b.len, in.size() - pos);
      std::memcpy(base + c * t->extent + b.disp, in.data() + pos, n);
      pos += n;
    }
  if (used) *used = pos;
  return true;
}

// Copy send-side elements into receive-side elements through the type maps.
int copy_typed(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount,
               MPI_Datatype rtype) {
  if (sbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  std::string bytes;
  if (!pack(sbuf, scount, stype, bytes)) return MPI_ERR_OTHER;
  if (!unpack(bytes, rbuf, rcount, rtype, nullptr)) return MPI_ERR_TRUNCATE;
  return MPI_SUCCESS;
}

struct CommRec {
  std::vector<int> graph_neighbours;
};
std::map<int, CommRec>& comms() {
  static std::map<int, CommRec> c = {{MPI_COMM_WORLD, {}}, {MPI_COMM_SELF, {}}};
  return c;
}
int next_comm = 3;

bool comm_ok(MPI_Comm c) { return comms().count(c) != 0; }

int next_group = 2;

struct Message {
  MPI_Comm comm;
  int tag;
  std::string bytes;
};
struct PendingRecv {
  int req;
  MPI_Comm comm;
  int tag;
  void* buf;
  int count;
  MPI_Datatype type;
};
struct ReqRec {
  bool done = false;
  MPI_Status status{0, 0, MPI_SUCCESS, 0};
};

std::deque<Message> queue_;
std::deque<PendingRecv> pending_;
std::map<int, ReqRec> requests_;
int next_req = 1;

bool tag_match(int want, int have) { return want == MPI_ANY_TAG || want == have; }

int new_request(bool done, int tag, long long bytes) {
  int id = next_req++;
  ReqRec r;
  r.done = done;
  r.status.MPI_TAG = tag;
  r.status.count_bytes = bytes;
  requests_[id] = r;
  return id;
}

// Deliver a packed message: to the oldest matching posted receive, else queue it.
int deliver(MPI_Comm comm, int tag, std::string&& bytes) {
  for (auto it = pending_.begin(); it != pending_.end(); ++it) {
    if (it->comm == comm && tag_match(it->tag, tag)) {
      size_t used = 0;
      if (!unpack(bytes, it->buf, it->count, it->type, &used)) return MPI_ERR_TRUNCATE;
      ReqRec& r = requests_[it->req];
      r.done = true;
      r.status.MPI_SOURCE = 0;
      r.status.MPI_TAG = tag;
      r.status.count_bytes = (long long)used;
      pending_.erase(it);
      return MPI_SUCCESS;
    }
  }
  queue_.push_back(Message{comm, tag, std::move(bytes)});
  return MPI_SUCCESS;
}

bool take(MPI_Comm comm, int tag, Message* out) {
  for (auto it = queue_.begin(); it != queue_.end(); ++it)
    if (it->comm == comm && tag_match(tag, it->tag)) {
      *out = std::move(*it);
      queue_.erase(it);
      return true;
    }
  return false;
}

struct FileRec {
  int fd = -1;
  MPI_Offset disp = 0;
  MPI_Datatype etype = MPI_BYTE;
  MPI_Offset pos = 0;         // individual pointer, etype units
  MPI_Offset shared_pos = 0;  // shared pointer, etype units
};
std::map<int, FileRec> files_;
int next_file = 1;

size_t etype_extent(const FileRec& f) {
  const TypeRec* t = type_of(f.etype);
  return t ? (size_t)t->extent : 1;
}

int file_read(FileRec& f, MPI_Offset off_bytes, void* buf, int count, MPI_Datatype type,
              MPI_Status* st) {
  const TypeRec* t = type_of(type);
  if (!t) return MPI_ERR_OTHER;
  std::string bytes(t->size * (size_t)count, '\0');
  size_t got = 0;
  while (got < bytes.size()) {
    ssize_t n = pread(f.fd, &bytes[got], bytes.size() - got, off_bytes + (MPI_Offset)got);
    if (n < 0) return MPI_ERR_FILE;
    if (n == 0) break;
    got += (size_t)n;
  }
  bytes.resize(got);
  size_t used = 0;
  if (!unpack(bytes, buf, count, type, &used)) return MPI_ERR_OTHER;
  if (st) {
    st->MPI_SOURCE = 0;
    st->MPI_TAG = 0;
    st->MPI_ERROR = MPI_SUCCESS;
    st->count_bytes = (long long)used;
  }
  return MPI_SUCCESS;
}

int file_write(FileRec& f, MPI_Offset off_bytes, const void* buf, int count, MPI_Datatype type,
               MPI_Status* st, size_t* written) {
  std::string bytes;
  if (!pack(buf, count, type, bytes)) return MPI_ERR_OTHER;
  size_t put = 0;
  while (put < bytes.size()) {
    ssize_t n = pwrite(f.fd, bytes.data() + put, bytes.size() - put, off_bytes + (MPI_Offset)put);
    if (n <= 0) return MPI_ERR_FILE;
    put += (size_t)n;
  }
  if (st) {
    st->MPI_SOURCE = 0;
    st->MPI_TAG = 0;
    st->MPI_ERROR = MPI_SUCCESS;
    st->count_bytes = (long long)put;
  }
  if (written) *written = put;
  return MPI_SUCCESS;
}

bool initialised = false;
bool finalised = false;

}  // namespace

extern "C" {

int MPI_Init(int*, char***) {
  initialised = true;
  return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) {
  *flag = initialised ? 1 : 0;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) {
  finalised = true;
  return MPI_SUCCESS;
}
int MPI_Finalized(int* flag) {
  *flag = finalised ? 1 : 0;
  return MPI_SUCCESS;
}
int MPI_Abort(MPI_Comm, int code) {
  std::fflush(nullptr);
  std::_Exit(code == 0 ? 1 : code);
}
double MPI_Wtime(void) {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Get_processor_name(char* name, int* len) {
  std::snprintf(name, MPI_MAX_PROCESSOR_NAME, "localhost");
  *len = (int)std::strlen(name);
  return MPI_SUCCESS;
}
int MPI_Error_string(int code, char* str, int* len) {
  std::snprintf(str, MPI_MAX_ERROR_STRING, "single-process MPI error %d", code);
  *len = (int)std::strlen(str);
  return MPI_SUCCESS;
}
int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int* size) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  *out = next_comm++;
  comms()[*out] = comms()[comm];
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm) {
  if (*comm != MPI_COMM_WORLD && *comm != MPI_COMM_SELF) comms().erase(*comm);
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result) {
  *result = a == b ? MPI_IDENT : MPI_CONGRUENT;
  return MPI_SUCCESS;
}
int MPI_Comm_group(MPI_Comm comm, MPI_Group* grp) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  *grp = next_group++;
  return MPI_SUCCESS;
}
static int comm_from_group(MPI_Comm comm, MPI_Group grp, MPI_Comm* out) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  if (grp == MPI_GROUP_EMPTY) {
    *out = MPI_COMM_NULL;
  } else {
    *out = next_comm++;
    comms()[*out] = CommRec{};
  }
  return MPI_SUCCESS;
}
int MPI_Comm_create(MPI_Comm comm, MPI_Group grp, MPI_Comm* out) { return comm_from_group(comm, grp, out); }
int MPI_Comm_create_group(MPI_Comm comm, MPI_Group grp, int, MPI_Comm* out) {
  return comm_from_group(comm, grp, out);
}
int MPI_Comm_split_type(MPI_Comm comm, int, int, MPI_Info, MPI_Comm* out) {
  return comm_from_group(comm, next_group++, out);
}
int MPI_Graph_create(MPI_Comm comm, int nnodes, const int index[], const int edges[], int, MPI_Comm* out) {
  if (!comm_ok(comm) || nnodes != 1) return MPI_ERR_OTHER;
  *out = next_comm++;
  CommRec r;
  for (int e = 0; e < index[0]; ++e) r.graph_neighbours.push_back(edges[e]);
  comms()[*out] = r;
  return MPI_SUCCESS;
}
int MPI_Graph_neighbors_count(MPI_Comm comm, int, int* n) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  *n = (int)comms()[comm].graph_neighbours.size();
  return MPI_SUCCESS;
}
int MPI_Graph_neighbors(MPI_Comm comm, int, int maxn, int neighbours[]) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  const auto& g = comms()[comm].graph_neighbours;
  for (int i = 0; i < maxn && i < (int)g.size(); ++i) neighbours[i] = g[i];
  return MPI_SUCCESS;
}

int MPI_Group_rank(MPI_Group grp, int* rank) {
  *rank = grp == MPI_GROUP_EMPTY ? MPI_UNDEFINED : 0;
  return MPI_SUCCESS;
}
int MPI_Group_size(MPI_Group grp, int* size) {
  *size = grp == MPI_GROUP_EMPTY ? 0 : 1;
  return MPI_SUCCESS;
}
int MPI_Group_incl(MPI_Group grp, int n, const int ranks[], MPI_Group* out) {
  if (n == 0 || grp == MPI_GROUP_EMPTY) {
    *out = MPI_GROUP_EMPTY;
    return MPI_SUCCESS;
  }
  if (n != 1 || ranks[0] != 0) return MPI_ERR_OTHER;
  *out = next_group++;
  return MPI_SUCCESS;
}
int MPI_Group_excl(MPI_Group grp, int n, const int ranks[], MPI_Group* out) {
  bool excl_self = false;
  for (int i = 0; i < n; ++i) excl_self |= ranks[i] == 0;
  *out = (excl_self || grp == MPI_GROUP_EMPTY) ? MPI_GROUP_EMPTY : next_group++;
  return MPI_SUCCESS;
}
int MPI_Group_free(MPI_Group* grp) {
  *grp = MPI_GROUP_NULL;
  return MPI_SUCCESS;
}

int MPI_Get_address(const void* location, MPI_Aint* address) {
  *address = (MPI_Aint)location;
  return MPI_SUCCESS;
}
int MPI_Type_create_struct(int count, const int blocklengths[], const MPI_Aint displacements[],
                           const MPI_Datatype tps[], MPI_Datatype* out) {
  TypeRec r;
  r.live = true;
  bool any = false;
  MPI_Aint lo = 0, hi = 0;
  for (int i = 0; i < count; ++i) {
    const TypeRec* t = type_of(tps[i]);
    if (!t) return MPI_ERR_OTHER;
    r.align = std::max(r.align, t->align);
    for (int j = 0; j < blocklengths[i]; ++j) {
      MPI_Aint base = displacements[i] + (MPI_Aint)j * t->extent;
      for (const Block& b : t->blocks) {
        Block nb{base + b.disp, b.len};
        if (!r.blocks.empty() && r.blocks.back().disp + (MPI_Aint)r.blocks.back().len == nb.disp)
          r.blocks.back().len += nb.len;
        else
          r.blocks.push_back(nb);
        r.size += b.len;
      }
      MPI_Aint l = base + t->lb, h = base + t->lb + t->extent;
      if (!any) {
        lo = l;
        hi = h;
        any = true;
      } else {
        lo = std::min(lo, l);
        hi = std::max(hi, h);
      }
    }
  }
  MPI_Aint ext = hi - lo;
  MPI_Aint a = (MPI_Aint)r.align;
  if (ext % a) ext += a - ext % a;
  r.lb = lo;
  r.extent = ext;
  types().push_back(r);
  *out = (MPI_Datatype)(types().size() - 1);
  return MPI_SUCCESS;
}
int MPI_Type_create_resized(MPI_Datatype type, MPI_Aint lb, MPI_Aint extent, MPI_Datatype* out) {
  const TypeRec* t = type_of(type);
  if (!t) return MPI_ERR_OTHER;
  TypeRec r = *t;
  r.lb = lb;
  r.extent = extent;
  types().push_back(r);
  *out = (MPI_Datatype)(types().size() - 1);
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype* type) { return type_of(*type) ? MPI_SUCCESS : MPI_ERR_OTHER; }
int MPI_Type_free(MPI_Datatype* type) {
  if (*type > MPI_BYTE && type_of(*type)) types()[*type].live = false;
  *type = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}
int MPI_Type_size(MPI_Datatype type, int* size) {
  const TypeRec* t = type_of(type);
  if (!t) return MPI_ERR_OTHER;
  *size = (int)t->size;
  return MPI_SUCCESS;
}
int MPI_Type_get_extent(MPI_Datatype type, MPI_Aint* lb, MPI_Aint* extent) {
  const TypeRec* t = type_of(type);
  if (!t) return MPI_ERR_OTHER;
  *lb = t->lb;
  *extent = t->extent;
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) { return comm_ok(comm) ? MPI_SUCCESS : MPI_ERR_OTHER; }
int MPI_Bcast(void*, int, MPI_Datatype type, int root, MPI_Comm comm) {
  return (comm_ok(comm) && root == 0 && type_of(type)) ? MPI_SUCCESS : MPI_ERR_OTHER;
}
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, int root,
               MPI_Comm comm) {
  if (!comm_ok(comm) || root != 0) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, count, type, recvbuf, count, type);
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm comm) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, count, type, recvbuf, count, type);
}
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
               MPI_Datatype recvtype, int root, MPI_Comm comm) {
  if (!comm_ok(comm) || root != 0) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
}
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                const int recvcounts[], const int displs[], MPI_Datatype recvtype, int root, MPI_Comm comm) {
  if (!comm_ok(comm) || root != 0) return MPI_ERR_OTHER;
  const TypeRec* t = type_of(recvtype);
  if (!t) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, sendcount, sendtype, (char*)recvbuf + displs[0] * t->extent, recvcounts[0],
                    recvtype);
}
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
}
int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                MPI_Datatype recvtype, int root, MPI_Comm comm) {
  if (!comm_ok(comm) || root != 0) return MPI_ERR_OTHER;
  if (recvbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  return copy_typed(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
}
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                 MPI_Datatype recvtype, MPI_Comm comm) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  return copy_typed(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
}
int MPI_Neighbor_allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                           int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  const auto& g = comms()[comm].graph_neighbours;
  const TypeRec* t = type_of(recvtype);
  if (!t) return MPI_ERR_OTHER;
  for (size_t i = 0; i < g.size(); ++i) {
    int rc = copy_typed(sendbuf, sendcount, sendtype, (char*)recvbuf + (MPI_Aint)i * recvcount * t->extent,
                        recvcount, recvtype);
    if (rc) return rc;
  }
  return MPI_SUCCESS;
}
int MPI_Neighbor_allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf,
                            const int recvcounts[], const int displs[], MPI_Datatype recvtype, MPI_Comm comm) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  const auto& g = comms()[comm].graph_neighbours;
  const TypeRec* t = type_of(recvtype);
  if (!t) return MPI_ERR_OTHER;
  for (size_t i = 0; i < g.size(); ++i) {
    int rc = copy_typed(sendbuf, sendcount, sendtype, (char*)recvbuf + displs[i] * t->extent, recvcounts[i],
                        recvtype);
    if (rc) return rc;
  }
  return MPI_SUCCESS;
}

int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request* req) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  if (dest == MPI_PROC_NULL) {
    *req = new_request(true, tag, 0);
    return MPI_SUCCESS;
  }
  if (dest != 0) return MPI_ERR_OTHER;
  std::string bytes;
  if (!pack(buf, count, type, bytes)) return MPI_ERR_OTHER;
  long long n = (long long)bytes.size();
  int rc = deliver(comm, tag, std::move(bytes));
  if (rc) return rc;
  *req = new_request(true, tag, n);
  return MPI_SUCCESS;
}
int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm) {
  MPI_Request r;
  int rc = MPI_Isend(buf, count, type, dest, tag, comm, &r);
  if (rc == MPI_SUCCESS) requests_.erase(r);
  return rc;
}
int MPI_Ssend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm) {
  return MPI_Send(buf, count, type, dest, tag, comm);
}
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  if (source == MPI_PROC_NULL) {
    *req = new_request(true, tag, 0);
    return MPI_SUCCESS;
  }
  if (source != 0 && source != MPI_ANY_SOURCE) return MPI_ERR_OTHER;
  Message m;
  if (take(comm, tag, &m)) {
    size_t used = 0;
    if (!unpack(m.bytes, buf, count, type, &used)) return MPI_ERR_TRUNCATE;
    *req = new_request(true, m.tag, (long long)used);
    return MPI_SUCCESS;
  }
  *req = new_request(false, tag, 0);
  pending_.push_back(PendingRecv{*req, comm, tag, buf, count, type});
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status* status) {
  if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
  auto it = requests_.find(*req);
  if (it == requests_.end()) return MPI_ERR_OTHER;
  if (!it->second.done) {
    // A receive from self with no matching send can never complete on one rank.
    std::fprintf(stderr, "single-process MPI: wait on an unmatched receive (tag %d)\n",
                 it->second.status.MPI_TAG);
    return MPI_ERR_OTHER;
  }
  if (status) *status = it->second.status;
  requests_.erase(it);
  *req = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status) {
  MPI_Request r;
  int rc = MPI_Irecv(buf, count, type, source, tag, comm, &r);
  if (rc) return rc;
  return MPI_Wait(&r, status);
}
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]) {
  for (int i = 0; i < count; ++i) {
    int rc = MPI_Wait(&reqs[i], statuses ? &statuses[i] : nullptr);
    if (rc) return rc;
  }
  return MPI_SUCCESS;
}
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* status) {
  if (*req == MPI_REQUEST_NULL) {
    *flag = 1;
    return MPI_SUCCESS;
  }
  auto it = requests_.find(*req);
  if (it == requests_.end()) return MPI_ERR_OTHER;
  *flag = it->second.done ? 1 : 0;
  if (*flag) return MPI_Wait(req, status);
  return MPI_SUCCESS;
}
int MPI_Testall(int count, MPI_Request reqs[], int* flag, MPI_Status statuses[]) {
  *flag = 1;
  for (int i = 0; i < count; ++i) {
    if (reqs[i] == MPI_REQUEST_NULL) continue;
    auto it = requests_.find(reqs[i]);
    if (it == requests_.end()) return MPI_ERR_OTHER;
    if (!it->second.done) *flag = 0;
  }
  if (*flag) return MPI_Waitall(count, reqs, statuses);
  return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status* status, MPI_Datatype type, int* count) {
  const TypeRec* t = type_of(type);
  if (!t || t->size == 0) return MPI_ERR_OTHER;
  *count = (int)(status->count_bytes / (long long)t->size);
  return MPI_SUCCESS;
}

int MPI_Info_create(MPI_Info* info) {
  *info = 1;
  return MPI_SUCCESS;
}
int MPI_Info_set(MPI_Info, const char*, const char*) { return MPI_SUCCESS; }
int MPI_Info_free(MPI_Info* info) {
  *info = MPI_INFO_NULL;
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm comm, const char* filename, int amode, MPI_Info, MPI_File* fh) {
  if (!comm_ok(comm)) return MPI_ERR_OTHER;
  int flags = 0;
  if (amode & MPI_MODE_RDWR)
    flags = O_RDWR;
  else if (amode & MPI_MODE_WRONLY)
    flags = O_WRONLY;
  else
    flags = O_RDONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  if (amode & MPI_MODE_EXCL) flags |= O_EXCL;
  int fd = open(filename, flags, 0644);
  if (fd < 0) return MPI_ERR_FILE;
  FileRec r;
  r.fd = fd;
  *fh = next_file++;
  files_[*fh] = r;
  return MPI_SUCCESS;
}
int MPI_File_close(MPI_File* fh) {
  auto it = files_.find(*fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  close(it->second.fd);
  files_.erase(it);
  *fh = MPI_FILE_NULL;
  return MPI_SUCCESS;
}
int MPI_File_get_size(MPI_File fh, MPI_Offset* size) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  struct stat st;
  if (fstat(it->second.fd, &st) != 0) return MPI_ERR_FILE;
  *size = (MPI_Offset)st.st_size;
  return MPI_SUCCESS;
}
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype, const char*,
                      MPI_Info) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  // Only contiguous file types occur in the reference (MPI_CHAR views).
  const TypeRec* ft = type_of(filetype);
  if (!ft || ft->blocks.size() != 1 || (size_t)ft->extent != ft->size) return MPI_ERR_OTHER;
  it->second.disp = disp;
  it->second.etype = etype;
  it->second.pos = 0;
  it->second.shared_pos = 0;
  return MPI_SUCCESS;
}
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void* buf, int count, MPI_Datatype type, MPI_Status* st) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  return file_read(f, f.disp + offset * (MPI_Offset)etype_extent(f), buf, count, type, st);
}
int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype type, MPI_Status* st) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  MPI_Status local;
  int rc = file_read(f, f.disp + f.pos * (MPI_Offset)etype_extent(f), buf, count, type, &local);
  if (rc) return rc;
  f.pos += local.count_bytes / (MPI_Offset)etype_extent(f);
  if (st) *st = local;
  return MPI_SUCCESS;
}
int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void* buf, int count, MPI_Datatype type,
                      MPI_Status* st) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  return file_write(f, f.disp + offset * (MPI_Offset)etype_extent(f), buf, count, type, st, nullptr);
}
int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype type, MPI_Status* st) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  size_t put = 0;
  int rc = file_write(f, f.disp + f.pos * (MPI_Offset)etype_extent(f), buf, count, type, st, &put);
  if (rc) return rc;
  f.pos += (MPI_Offset)(put / etype_extent(f));
  return MPI_SUCCESS;
}
int MPI_File_write_ordered(MPI_File fh, const void* buf, int count, MPI_Datatype type, MPI_Status* st) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  size_t put = 0;
  int rc = file_write(f, f.disp + f.shared_pos * (MPI_Offset)etype_extent(f), buf, count, type, st, &put);
  if (rc) return rc;
  f.shared_pos += (MPI_Offset)(put / etype_extent(f));
  return MPI_SUCCESS;
}
int MPI_File_seek_shared(MPI_File fh, MPI_Offset offset, int whence) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  FileRec& f = it->second;
  if (whence == MPI_SEEK_SET) {
    f.shared_pos = offset;
  } else if (whence == MPI_SEEK_CUR) {
    f.shared_pos += offset;
  } else {
    MPI_Offset size = 0;
    MPI_File_get_size(fh, &size);
    f.shared_pos = (size - f.disp) / (MPI_Offset)etype_extent(f) + offset;
  }
  return MPI_SUCCESS;
}
int MPI_File_get_position_shared(MPI_File fh, MPI_Offset* offset) {
  auto it = files_.find(fh);
  if (it == files_.end()) return MPI_ERR_FILE;
  *offset = it->second.shared_pos;
  return MPI_SUCCESS;
}

int MPI_Win_allocate_shared(MPI_Aint size, int, MPI_Info, MPI_Comm, void* baseptr, MPI_Win* win) {
  void* p = std::calloc(size > 0 ? (size_t)size : 1, 1);
  if (!p) return MPI_ERR_OTHER;
  *(void**)baseptr = p;
  static std::map<int, void*> wins;
  static int next = 1;
  *win = next++;
  wins[*win] = p;
  return MPI_SUCCESS;
}
int MPI_Win_shared_query(MPI_Win, int, MPI_Aint*, int*, void*) { return MPI_ERR_OTHER; }
int MPI_Win_fence(int, MPI_Win) { return MPI_SUCCESS; }
int MPI_Win_free(MPI_Win* win) {
  *win = MPI_WIN_NULL;
  return MPI_SUCCESS;
}

}  // extern "C"
