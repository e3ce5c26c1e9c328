// Test infrastructure for the oracle build of the reference (not product code).
//
// A minimal MPI for running the reference's np ranks as forked processes on
// one host.  Every pair of ranks shares a socketpair.  Writes never block
// forever: while a rank waits to write (or to receive), it keeps draining all
// incoming sockets into per-peer inboxes, so two ranks that send to each other
// at the same time cannot deadlock.  A rank whose peer dies exits with an
// error; SNU_MPI_TIMEOUT (seconds, default 7200) bounds the whole run.
#include "mpi.h"

#include <errno.h>
#include <poll.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/socket.h>
#include <sys/time.h>
#include <sys/wait.h>
#include <unistd.h>

#include <deque>
#include <vector>

namespace {

struct Msg {
  int tag;
  std::vector<char> data;
};

struct Peer {
  int fd = -1;
  bool closed = false;  // the peer exited (normal at finalize)
  std::vector<char> in;  // bytes read but not yet parsed
  std::deque<Msg> inbox;
};

int g_rank = 0, g_size = 1;
std::vector<Peer> g_peer;
std::vector<pid_t> g_children;

const int TAG_BCAST = -101, TAG_SCATTER = -102, TAG_GATHER = -103,
          TAG_BARRIER = -104, TAG_FIN = -105;

void die(const char* what) {
  fprintf(stderr, "[mini-mpi rank %d] fatal: %s (errno %d)\n", g_rank, what,
          errno);
  fflush(stderr);
  if (g_rank == 0)
    for (pid_t c : g_children) kill(c, SIGKILL);
  _exit(3);
}

size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_INT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_BYTE: return 1;
    case MPI_FLOAT: return 4;
    case MPI_INT64_T: return 8;
    case MPI_CHAR: return 1;
    default: return 1;
  }
}

struct Header {
  int tag;
  int pad;
  long long bytes;
};

void parse(Peer& p) {
  size_t off = 0;
  while (p.in.size() - off >= sizeof(Header)) {
    Header h;
    memcpy(&h, p.in.data() + off, sizeof h);
    if (p.in.size() - off - sizeof h < (size_t)h.bytes) break;
    Msg m;
    m.tag = h.tag;
    m.data.assign(p.in.begin() + off + sizeof h,
                  p.in.begin() + off + sizeof h + h.bytes);
    p.inbox.push_back(std::move(m));
    off += sizeof h + h.bytes;
  }
  if (off) p.in.erase(p.in.begin(), p.in.begin() + off);
}

// Reads whatever is available on one socket.
void drain(int peer) {
  char buf[1 << 16];
  for (;;) {
    ssize_t r = recv(g_peer[peer].fd, buf, sizeof buf, MSG_DONTWAIT);
    if (r > 0) {
      g_peer[peer].in.insert(g_peer[peer].in.end(), buf, buf + r);
      continue;
    }
    if (r == 0) {
      g_peer[peer].closed = true;  // only fatal if we still need its data
      break;
    }
    if (errno == EAGAIN || errno == EWOULDBLOCK) break;
    if (errno == EINTR) continue;
    die("recv failed");
  }
  parse(g_peer[peer]);
}

// Polls every peer socket for input (and optionally one for output).
// Returns true when the output socket is writable.
bool progress(int out_peer, int timeout_ms) {
  std::vector<pollfd> fds;
  std::vector<int> who;
  for (int r = 0; r < g_size; r++) {
    if (r == g_rank || g_peer[r].closed) continue;
    pollfd p{g_peer[r].fd, POLLIN, 0};
    if (r == out_peer) p.events |= POLLOUT;
    fds.push_back(p);
    who.push_back(r);
  }
  if (fds.empty()) return out_peer < 0 ? false : true;
  int rc = poll(fds.data(), fds.size(), timeout_ms);
  if (rc < 0) {
    if (errno == EINTR) return false;
    die("poll failed");
  }
  bool writable = false;
  for (size_t k = 0; k < fds.size(); k++) {
    if (fds[k].revents & (POLLIN | POLLHUP | POLLERR)) drain(who[k]);
    if (who[k] == out_peer && (fds[k].revents & POLLOUT)) writable = true;
  }
  return writable;
}

void send_bytes(int dest, int tag, const void* buf, long long bytes) {
  if (dest == g_rank) {
    Msg m;
    m.tag = tag;
    m.data.assign((const char*)buf, (const char*)buf + bytes);
    g_peer[dest].inbox.push_back(std::move(m));
    return;
  }
  if (g_peer[dest].closed) die("send to a rank that exited");
  Header h{tag, 0, bytes};
  std::vector<char> out(sizeof h + bytes);
  memcpy(out.data(), &h, sizeof h);
  if (bytes) memcpy(out.data() + sizeof h, buf, bytes);
  size_t done = 0;
  while (done < out.size()) {
    ssize_t w = send(g_peer[dest].fd, out.data() + done, out.size() - done,
                     MSG_DONTWAIT | MSG_NOSIGNAL);
    if (w > 0) {
      done += (size_t)w;
      continue;
    }
    if (w < 0 && errno != EAGAIN && errno != EWOULDBLOCK && errno != EINTR)
      die("send failed");
    progress(dest, 1000);
  }
}

void recv_bytes(int src, int tag, void* buf, long long max_bytes) {
  for (;;) {
    auto& box = g_peer[src].inbox;
    for (auto it = box.begin(); it != box.end(); ++it) {
      if (it->tag == tag) {
        long long n = (long long)it->data.size();
        if (n > max_bytes) die("message larger than the receive buffer");
        if (n) memcpy(buf, it->data.data(), n);
        box.erase(it);
        return;
      }
    }
    if (src == g_rank) die("self receive without a matching send");
    if (g_peer[src].closed) die("peer exited before sending a message");
    progress(-1, 1000);
  }
}

void on_alarm(int) { die("SNU_MPI_TIMEOUT expired"); }

}  // namespace

extern "C" {

int MPI_Init(int*, char***) {
  const char* e = getenv("SNU_MPI_NP");
  g_size = e ? atoi(e) : 1;
  if (g_size < 1) g_size = 1;
  const char* to = getenv("SNU_MPI_TIMEOUT");
  signal(SIGALRM, on_alarm);
  alarm(to ? atoi(to) : 7200);
  // socketpair for every pair (i < j): fd i-side, j-side
  std::vector<std::vector<int>> fd(g_size, std::vector<int>(g_size, -1));
  for (int i = 0; i < g_size; i++)
    for (int j = i + 1; j < g_size; j++) {
      int sv[2];
      if (socketpair(AF_UNIX, SOCK_STREAM, 0, sv) != 0) die("socketpair");
      int sz = 4 << 20;
      setsockopt(sv[0], SOL_SOCKET, SO_SNDBUF, &sz, sizeof sz);
      setsockopt(sv[1], SOL_SOCKET, SO_SNDBUF, &sz, sizeof sz);
      fd[i][j] = sv[0];
      fd[j][i] = sv[1];
    }
  fflush(stdout);
  fflush(stderr);
  g_rank = 0;
  for (int r = 1; r < g_size; r++) {
    pid_t pid = fork();
    if (pid < 0) die("fork");
    if (pid == 0) {
      g_rank = r;
      g_children.clear();
      break;
    }
    g_children.push_back(pid);
  }
  g_peer.assign(g_size, Peer());
  for (int i = 0; i < g_size; i++)
    for (int j = 0; j < g_size; j++) {
      if (i == j || fd[i][j] < 0) continue;
      if (i == g_rank)
        g_peer[j].fd = fd[i][j];
      else
        close(fd[i][j]);
    }
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  MPI_Barrier(MPI_COMM_WORLD);
  fflush(stdout);
  fflush(stderr);
  if (g_rank != 0) _exit(0);
  int bad = 0;
  for (pid_t c : g_children) {
    int st = 0;
    waitpid(c, &st, 0);
    if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
  }
  if (bad) {
    fprintf(stderr, "[mini-mpi] a rank failed\n");
    _exit(4);
  }
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = g_rank;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int* s) {
  *s = g_size;
  return MPI_SUCCESS;
}

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag,
             MPI_Comm) {
  send_bytes(dest, tag, buf, (long long)count * type_size(t));
  return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm,
             MPI_Status* st) {
  recv_bytes(src, tag, buf, (long long)count * type_size(t));
  if (st) st->MPI_SOURCE = src, st->MPI_TAG = tag, st->MPI_ERROR = 0;
  return MPI_SUCCESS;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag,
              MPI_Comm c, MPI_Request* req) {
  MPI_Send(buf, count, t, dest, tag, c);  // eager: complete at once
  req->kind = 0;
  return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm,
              MPI_Request* req) {
  req->kind = 1;
  req->buf = buf;
  req->bytes = (long long)count * type_size(t);
  req->peer = src;
  req->tag = tag;
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status* st) {
  if (req->kind == 1) {
    recv_bytes(req->peer, req->tag, req->buf, req->bytes);
    req->kind = 0;
  }
  if (st) st->MPI_ERROR = 0;
  return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm) {
  long long b = (long long)count * type_size(t);
  if (g_rank == root) {
    for (int r = 0; r < g_size; r++)
      if (r != root) send_bytes(r, TAG_BCAST, buf, b);
  } else {
    recv_bytes(root, TAG_BCAST, buf, b);
  }
  return MPI_SUCCESS;
}

int MPI_Scatterv(const void* sendbuf, const int* counts, const int* displs,
                 MPI_Datatype st, void* recvbuf, int recvcount,
                 MPI_Datatype rt, int root, MPI_Comm) {
  if (g_rank == root) {
    size_t es = type_size(st);
    for (int r = 0; r < g_size; r++) {
      const char* p = (const char*)sendbuf + (size_t)displs[r] * es;
      if (r == root)
        memcpy(recvbuf, p, (size_t)counts[r] * es);
      else
        send_bytes(r, TAG_SCATTER, p, (long long)counts[r] * es);
    }
  } else {
    recv_bytes(root, TAG_SCATTER, recvbuf, (long long)recvcount * type_size(rt));
  }
  return MPI_SUCCESS;
}

int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype st,
                void* recvbuf, int recvcount, MPI_Datatype rt, int root,
                MPI_Comm c) {
  std::vector<int> counts(g_size, sendcount), displs(g_size);
  for (int r = 0; r < g_size; r++) displs[r] = r * sendcount;
  return MPI_Scatterv(sendbuf, counts.data(), displs.data(), st, recvbuf,
                      recvcount, rt, root, c);
}

int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype st,
                void* recvbuf, const int* counts, const int* displs,
                MPI_Datatype rt, int root, MPI_Comm) {
  if (g_rank == root) {
    size_t es = type_size(rt);
    for (int r = 0; r < g_size; r++) {
      char* p = (char*)recvbuf + (size_t)displs[r] * es;
      if (r == root)
        memcpy(p, sendbuf, (size_t)sendcount * type_size(st));
      else
        recv_bytes(r, TAG_GATHER, p, (long long)counts[r] * es);
    }
  } else {
    send_bytes(root, TAG_GATHER, sendbuf, (long long)sendcount * type_size(st));
  }
  return MPI_SUCCESS;
}

int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype st,
               void* recvbuf, int recvcount, MPI_Datatype rt, int root,
               MPI_Comm c) {
  std::vector<int> counts(g_size, recvcount), displs(g_size);
  for (int r = 0; r < g_size; r++) displs[r] = r * recvcount;
  return MPI_Gatherv(sendbuf, sendcount, st, recvbuf, counts.data(),
                     displs.data(), rt, root, c);
}

int MPI_Barrier(MPI_Comm) {
  char token = 0;
  if (g_rank == 0) {
    for (int r = 1; r < g_size; r++) recv_bytes(r, TAG_BARRIER, &token, 1);
    for (int r = 1; r < g_size; r++) send_bytes(r, TAG_BARRIER, &token, 1);
  } else {
    send_bytes(0, TAG_BARRIER, &token, 1);
    recv_bytes(0, TAG_BARRIER, &token, 1);
  }
  return MPI_SUCCESS;
}

double MPI_Wtime(void) {
  timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

}  // extern "C"

// TAG_FIN is reserved for future use by the harness.
static_assert(TAG_FIN < 0, "reserved tags are negative");
