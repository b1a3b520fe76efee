/*
 * mpi.h -- in-process MPI stand-in used only to compile the reference
 * sources as a test checker (oracle/build_ref.sh).  Ranks are threads of one
 * process; each thread sets its rank with ippi_mpi_enter().  Only the calls
 * the reference makes are provided: Init/Comm_rank/Comm_size/Finalize,
 * Barrier, blocking Send/Recv (buffered: Send never waits), Allreduce(SUM,
 * double) and Abort (throws ippi_mpi_abort so the driver can report it).
 * With one rank, Send/Recv to self reproduce the reference's periodic ring.
 */
#ifndef IPPI_REF_MPI_SHIM_H
#define IPPI_REF_MPI_SHIM_H

#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_FLOAT 2
#define MPI_INT 3
#define MPI_SUM 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

struct ippi_mpi_abort : std::runtime_error {
    explicit ippi_mpi_abort(int c) : std::runtime_error("MPI_Abort"), code(c) {}
    int code;
};

struct ippi_mpi_world {
    int size = 1;
    std::mutex mu;
    std::condition_variable cv;
    std::map<std::tuple<int, int, int>, std::deque<std::vector<char>>> box;
    int bar_count = 0;
    long bar_gen = 0;
    std::vector<double> red;
    int red_count = 0;
    long red_gen = 0;
    bool aborted = false;
};

inline ippi_mpi_world*& ippi_mpi_world_ptr()
{
    static ippi_mpi_world* w = nullptr;
    return w;
}
inline int& ippi_mpi_rank()
{
    static thread_local int r = 0;
    return r;
}
inline void ippi_mpi_enter(ippi_mpi_world* w, int rank)
{
    ippi_mpi_world_ptr() = w;
    ippi_mpi_rank() = rank;
}

inline size_t ippi_mpi_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = ippi_mpi_rank(); return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = ippi_mpi_world_ptr()->size; return 0; }

inline int MPI_Abort(MPI_Comm, int code)
{
    ippi_mpi_world* w = ippi_mpi_world_ptr();
    {
        std::lock_guard<std::mutex> g(w->mu);
        w->aborted = true;
    }
    w->cv.notify_all();
    throw ippi_mpi_abort(code);
}

inline int MPI_Barrier(MPI_Comm)
{
    ippi_mpi_world* w = ippi_mpi_world_ptr();
    std::unique_lock<std::mutex> g(w->mu);
    long gen = w->bar_gen;
    if (++w->bar_count == w->size) {
        w->bar_count = 0;
        w->bar_gen++;
        w->cv.notify_all();
    } else {
        w->cv.wait(g, [&] { return w->bar_gen != gen || w->aborted; });
        if (w->aborted) throw ippi_mpi_abort(1);
    }
    return 0;
}

inline int MPI_Send(const void* buf, int n, MPI_Datatype t, int dst, int tag, MPI_Comm)
{
    ippi_mpi_world* w = ippi_mpi_world_ptr();
    std::vector<char> m((size_t)n * ippi_mpi_size(t));
    if (n) std::memcpy(m.data(), buf, m.size());
    /* the reference's ring sends rank 0 -> RankID+1 even with one rank
     * (mesh.cpp:468); ranks wrap around the ring */
    dst = ((dst % w->size) + w->size) % w->size;
    {
        std::lock_guard<std::mutex> g(w->mu);
        w->box[std::make_tuple(ippi_mpi_rank(), dst, tag)].push_back(std::move(m));
    }
    w->cv.notify_all();
    return 0;
}

inline int MPI_Recv(void* buf, int n, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status*)
{
    ippi_mpi_world* w = ippi_mpi_world_ptr();
    src = ((src % w->size) + w->size) % w->size;
    std::unique_lock<std::mutex> g(w->mu);
    auto key = std::make_tuple(src, ippi_mpi_rank(), tag);
    w->cv.wait(g, [&] { return !w->box[key].empty() || w->aborted; });
    if (w->aborted) throw ippi_mpi_abort(1);
    std::vector<char> m = std::move(w->box[key].front());
    w->box[key].pop_front();
    size_t bytes = (size_t)n * ippi_mpi_size(t);
    std::memcpy(buf, m.data(), bytes < m.size() ? bytes : m.size());
    return 0;
}

inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    ippi_mpi_world* w = ippi_mpi_world_ptr();
    std::unique_lock<std::mutex> g(w->mu);
    long gen = w->red_gen;
    if (w->red_count == 0) w->red.assign((size_t)n, 0.0);
    for (int i = 0; i < n; i++)
        w->red[i] += (t == MPI_DOUBLE) ? ((const double*)in)[i] : ((const float*)in)[i];
    if (++w->red_count == w->size) {
        w->red_count = 0;
        w->red_gen++;
        w->cv.notify_all();
    } else {
        w->cv.wait(g, [&] { return w->red_gen != gen || w->aborted; });
        if (w->aborted) throw ippi_mpi_abort(1);
    }
    for (int i = 0; i < n; i++) {
        if (t == MPI_DOUBLE) ((double*)out)[i] = w->red[i];
        else ((float*)out)[i] = (float)w->red[i];
    }
    return 0;
}

#endif
