// Frame output for a simulation loop: the datasets and the XDMF time-series
// index of the reference's HDF5Exporter (io/hdf5_exporter.cpp:10-128),
// with the datasets stored as raw little-endian FP64 in one file per frame
// (XDMF "Binary" data items with byte offsets) instead of HDF5.
//
// Frames from device arrays: a device-to-device snapshot on the caller's
// stream (microseconds), then the copy of the snapshot into page-locked
// staging on a copy stream of this writer, and the file written by a writer
// thread once that copy has completed.  The caller's next steps may change
// its arrays at once; the host copy and the file writing overlap them.  Two
// slots; frames are written in call order.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "fmm_gpu.h"

struct fmm_frames {
  std::string dir, base;
  int dim = 3;
  // frames written so far, for the index: time, file name, particle count
  std::vector<double> times;
  std::vector<std::string> names;
  std::vector<int64_t> counts;

  struct Slot {
    double *buf = nullptr;  // page-locked: positions, velocities, accelerations (n x dim each), masses
    double *dbuf = nullptr; // the device snapshot, same layout
    size_t cap = 0;         // doubles
    cudaEvent_t snap = nullptr, done = nullptr;
    bool busy = false;
    bool has_acc = true;
    int64_t n = 0;
    int step = 0;
    double time = 0.0;
  };
  Slot slots[2];
  int next_slot = 0;
  int device = -1;             // the device of the device frames (set by the first)
  cudaStream_t copy = nullptr; // the host copies of the snapshots

  std::mutex mu;
  std::condition_variable cv;
  std::deque<int> queue;  // slots waiting for the writer, in call order
  int writing = -1;       // the slot the writer holds
  bool stop = false;
  int err = FMM_OK;
  std::thread writer;
};

namespace {

std::string frame_name(const fmm_frames *f, int step) {
  char num[32];
  std::snprintf(num, sizeof(num), "%05d", step);  // std::setw(5) << setfill('0'), hdf5_exporter.cpp:17
  return f->base + "_" + num + ".bin";
}

// The index, rewritten after every frame (hdf5_exporter.cpp:83-128); each
// step's grid carries its own particle count, and its data items point at
// the datasets inside that step's .bin file.
int write_index(const fmm_frames *f) {
  const std::string path = f->dir + "/" + f->base + ".xmf";
  std::ofstream x(path);
  if (!x.is_open()) return FMM_ERR_IO;
  x << "<?xml version=\"1.0\" ?>\n";
  x << "<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n";
  x << "<Xdmf Version=\"2.0\">\n";
  x << " <Domain>\n";
  x << "  <Grid Name=\"TimeSeries\" GridType=\"Collection\" CollectionType=\"Temporal\">\n";
  for (size_t t = 0; t < f->times.size(); ++t) {
    const int64_t n = f->counts[t];
    const std::string &file = f->names[t];
    auto item = [&](const char *dims, int64_t seek) {
      x << "       <DataItem Dimensions=\"" << dims << "\" NumberType=\"Float\" Precision=\"8\" Format=\"Binary\""
        << " Endian=\"Little\" Seek=\"" << seek << "\">\n";
      x << "         " << file << "\n";
      x << "       </DataItem>\n";
    };
    const std::string d3 = std::to_string(n) + " 3", d1 = std::to_string(n);
    x << "   <Grid Name=\"Step_" << t << "\" GridType=\"Uniform\">\n";
    x << "     <Time Value=\"" << f->times[t] << "\"/>\n";
    x << "     <Topology TopologyType=\"Polyvertex\" NumberOfElements=\"" << n << "\"/>\n";
    x << "     <Geometry GeometryType=\"XYZ\">\n";
    item(d3.c_str(), 0);
    x << "     </Geometry>\n";
    x << "     <Attribute Name=\"Velocity\" AttributeType=\"Vector\" Center=\"Node\">\n";
    item(d3.c_str(), 24 * n);
    x << "     </Attribute>\n";
    x << "     <Attribute Name=\"Acceleration\" AttributeType=\"Vector\" Center=\"Node\">\n";
    item(d3.c_str(), 48 * n);
    x << "     </Attribute>\n";
    x << "     <Attribute Name=\"Weight\" AttributeType=\"Scalar\" Center=\"Node\">\n";
    item(d1.c_str(), 72 * n);
    x << "     </Attribute>\n";
    x << "   </Grid>\n";
  }
  x << "  </Grid>\n";
  x << " </Domain>\n";
  x << "</Xdmf>\n";
  x.close();
  return x.fail() ? FMM_ERR_IO : FMM_OK;
}

// One frame: the three vector datasets padded to 3 components
// (hdf5_exporter.cpp:29-44), then the weights; then the index.  The caller
// holds no lock; only the writer thread or a synchronous write (after a
// flush) runs this, so frames stay in order.
int write_frame_unguarded(fmm_frames *f, int64_t n, const double *pos, const double *vel, const double *acc,
                const double *mass, int step, double time) {
  if (n <= 0) return FMM_OK;  // hdf5_exporter.cpp:22
  const int dim = f->dim;
  const std::string name = frame_name(f, step);
  FILE *fp = std::fopen((f->dir + "/" + name).c_str(), "wb");
  if (!fp) return FMM_ERR_IO;
  std::vector<double> row;
  const size_t chunk = 1 << 16;  // particles per buffered write
  row.resize(chunk * 3);
  bool ok = true;
  for (int set = 0; set < 3 && ok; ++set) {
    const double *src = set == 0 ? pos : set == 1 ? vel : acc;
    for (int64_t i0 = 0; i0 < n && ok; i0 += (int64_t)chunk) {
      const int64_t m = std::min<int64_t>((int64_t)chunk, n - i0);
      for (int64_t i = 0; i < m; ++i)
        for (int k = 0; k < 3; ++k) row[3 * i + k] = (src && k < dim) ? src[(i0 + i) * dim + k] : 0.0;
      ok = std::fwrite(row.data(), sizeof(double), (size_t)(3 * m), fp) == (size_t)(3 * m);
    }
  }
  if (ok) ok = std::fwrite(mass, sizeof(double), (size_t)n, fp) == (size_t)n;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) return FMM_ERR_IO;
  f->times.push_back(time);
  f->names.push_back(name);
  f->counts.push_back(n);
  return write_index(f);
}

// The same with allocation failures (strings, buffers, the frame lists)
// turned into a status: nothing may throw across the C ABI or out of the
// writer thread.
int write_frame(fmm_frames *f, int64_t n, const double *pos, const double *vel, const double *acc,
                const double *mass, int step, double time) {
  try {
    return write_frame_unguarded(f, n, pos, vel, acc, mass, step, time);
  } catch (const std::bad_alloc &) {
    return FMM_ERR_OUT_OF_MEMORY;
  } catch (...) {
    return FMM_ERR_INTERNAL;
  }
}

void writer_loop(fmm_frames *f) {
  std::unique_lock<std::mutex> lk(f->mu);
  while (true) {
    f->cv.wait(lk, [&] { return f->stop || !f->queue.empty(); });
    if (f->queue.empty()) return;  // stop, nothing left
    const int s = f->queue.front();
    f->queue.pop_front();
    f->writing = s;
    fmm_frames::Slot &sl = f->slots[s];
    lk.unlock();
    int rc = FMM_OK;
    if (cudaSetDevice(f->device) != cudaSuccess || cudaEventSynchronize(sl.done) != cudaSuccess) rc = FMM_ERR_CUDA;
    if (rc == FMM_OK) {
      const size_t nd = (size_t)sl.n * f->dim;
      rc = write_frame(f, sl.n, sl.buf, sl.buf + nd, sl.has_acc ? sl.buf + 2 * nd : nullptr, sl.buf + 3 * nd, sl.step,
                       sl.time);
    }
    lk.lock();
    if (rc != FMM_OK && f->err == FMM_OK) f->err = rc;
    sl.busy = false;
    f->writing = -1;
    f->cv.notify_all();
  }
}

// Waits (lock held) until no frame is queued or being written.
void wait_idle(fmm_frames *f, std::unique_lock<std::mutex> &lk) {
  f->cv.wait(lk, [&] { return f->queue.empty() && f->writing < 0; });
}

}  // namespace

extern "C" {

int fmm_frames_open(const char *dir, const char *base, int32_t dim, fmm_frames **out) {
  if (!dir || !base || !out || (dim != 2 && dim != 3) || !*base) return FMM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (mkdir(dir, 0755) != 0 && errno != EEXIST) return FMM_ERR_IO;  // hdf5_exporter.cpp:12
  fmm_frames *f = new (std::nothrow) fmm_frames;
  if (!f) return FMM_ERR_OUT_OF_MEMORY;
  try {
    f->dir = dir;
    f->base = base;
    f->dim = dim;
    f->writer = std::thread(writer_loop, f);
  } catch (...) {
    delete f;
    return FMM_ERR_INTERNAL;
  }
  *out = f;
  return FMM_OK;
}

int fmm_frames_write(fmm_frames *f, int64_t n, const double *pos, const double *vel, const double *acc,
                     const double *mass, int32_t step, double time) {
  if (!f || n < 0 || step < 0 || (n > 0 && (!pos || !vel || !mass))) return FMM_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(f->mu);
  wait_idle(f, lk);  // frames in flight first: the index lists frames in call order
  const int rc = write_frame(f, n, pos, vel, acc, mass, step, time);
  if (rc != FMM_OK && f->err == FMM_OK) f->err = rc;
  return rc;
}

int fmm_frames_write_device(fmm_frames *f, int64_t n, const double *d_pos, const double *d_vel, const double *d_acc,
                            const double *d_mass, int32_t step, double time, void *stream) {
  if (!f || n < 0 || step < 0 || (n > 0 && (!d_pos || !d_vel || !d_mass))) return FMM_ERR_INVALID_ARGUMENT;
  if (n == 0) return FMM_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FMM_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  std::unique_lock<std::mutex> lk(f->mu);
  if (f->device >= 0 && f->device != dev) return FMM_ERR_INVALID_ARGUMENT;  // one device per writer
  if (!f->copy) {
    if (cudaStreamCreateWithFlags(&f->copy, cudaStreamNonBlocking) != cudaSuccess) {
      f->copy = nullptr;
      return FMM_ERR_CUDA;
    }
    f->device = dev;
  }
  const int s = f->next_slot;
  fmm_frames::Slot &sl = f->slots[s];
  f->cv.wait(lk, [&] { return !sl.busy; });  // at most two frames in flight
  if (f->err != FMM_OK) return f->err;
  const size_t nd = (size_t)n * f->dim, need = 3 * nd + (size_t)n;
  if (sl.cap < need) {
    if (sl.buf) cudaFreeHost(sl.buf);
    if (sl.dbuf) cudaFree(sl.dbuf);
    sl.buf = nullptr;
    sl.dbuf = nullptr;
    sl.cap = 0;
    if (cudaHostAlloc((void **)&sl.buf, need * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
      sl.buf = nullptr;
      return FMM_ERR_OUT_OF_MEMORY;
    }
    if (cudaMalloc((void **)&sl.dbuf, need * sizeof(double)) != cudaSuccess) {
      sl.dbuf = nullptr;
      return FMM_ERR_OUT_OF_MEMORY;
    }
    sl.cap = need;
  }
  if ((!sl.snap && cudaEventCreateWithFlags(&sl.snap, cudaEventDisableTiming) != cudaSuccess) ||
      (!sl.done && cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess))
    return FMM_ERR_CUDA;
  const size_t vb = nd * sizeof(double);
  // the snapshot, ordered after the caller's work on `stream`
  if (cudaMemcpyAsync(sl.dbuf, d_pos, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(sl.dbuf + nd, d_vel, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      (d_acc && cudaMemcpyAsync(sl.dbuf + 2 * nd, d_acc, vb, cudaMemcpyDeviceToDevice, st) != cudaSuccess) ||
      cudaMemcpyAsync(sl.dbuf + 3 * nd, d_mass, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st) !=
          cudaSuccess ||
      cudaEventRecord(sl.snap, st) != cudaSuccess)
    return FMM_ERR_CUDA;
  // its host copy on the writer's stream
  if (cudaStreamWaitEvent(f->copy, sl.snap, 0) != cudaSuccess ||
      cudaMemcpyAsync(sl.buf, sl.dbuf, need * sizeof(double), cudaMemcpyDeviceToHost, f->copy) != cudaSuccess ||
      cudaEventRecord(sl.done, f->copy) != cudaSuccess)
    return FMM_ERR_CUDA;
  sl.busy = true;
  sl.has_acc = d_acc != nullptr;
  sl.n = n;
  sl.step = step;
  sl.time = time;
  f->queue.push_back(s);
  f->next_slot ^= 1;
  f->cv.notify_all();
  return FMM_OK;
}

int fmm_frames_flush(fmm_frames *f) {
  if (!f) return FMM_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(f->mu);
  wait_idle(f, lk);
  return f->err;
}

int fmm_frames_close(fmm_frames *f) {
  if (!f) return FMM_ERR_INVALID_ARGUMENT;
  int rc;
  {
    std::unique_lock<std::mutex> lk(f->mu);
    wait_idle(f, lk);
    rc = f->err;
    f->stop = true;
    f->cv.notify_all();
  }
  f->writer.join();
  if (f->device >= 0) cudaSetDevice(f->device);
  for (auto &sl : f->slots) {
    if (sl.buf) cudaFreeHost(sl.buf);
    if (sl.dbuf) cudaFree(sl.dbuf);
    if (sl.snap) cudaEventDestroy(sl.snap);
    if (sl.done) cudaEventDestroy(sl.done);
  }
  if (f->copy) cudaStreamDestroy(f->copy);
  delete f;
  return rc;
}

}  // extern "C"
