// algs.cuh - scaffolding for graph algorithms written against the cuStinger algorithm library
// (the reference's include/algs.cuh interface, used by its BFS, connected components and
// PageRank under src/static_*): the StaticAlgorithm interface, a device work queue, and the
// signatures of the per-vertex and per-edge functions that the traversal operators
// (operators.cuh) call.
#ifndef CUSTINGER_ALGS_CUH_
#define CUSTINGER_ALGS_CUH_

#include <cuda_runtime.h>

#include "cuStinger.hpp"
#include "utils.hpp"

namespace cuStingerAlgs {

// A per-vertex function f(custing, v, metadata) and a per-edge function f(custing, src, dst,
// metadata): __device__ functions passed to the operators as template arguments, so each
// traversal kernel inlines its function.
typedef void (*cusSubKernelVertex)(cuStinger* custing, vertexId_t src, void* metadata);
typedef void (*cusSubKernelEdge)(cuStinger* custing, vertexId_t src, vertexId_t dst, void* metadata);

class StaticAlgorithm {
 public:
  virtual void Init(cuStinger& custing) = 0;
  virtual void Reset() = 0;
  virtual void Run(cuStinger& custing) = 0;
  virtual void Release() = 0;
  virtual void SyncHostWithDevice() = 0;
  virtual void SyncDeviceWithHost() = 0;
};

// A device array with a consumed prefix [0, queueCurr) and an active part [queueCurr, queueEnd).
// Kernels append with enqueue() on a device copy of the object: either a copy inside an
// algorithm's metadata struct (copied to the device and back as plain bytes) or the one that
// devPtr() returns (SyncHostWithDevice / SyncDeviceWithHost move the indices between them).
template <class T>
class Queue {
 public:
  Queue() {}
  explicit Queue(length_t length) { Init(length); }
  ~Queue() { release(); }
  // The queue owns its device arrays: no C++ copies (algorithms move it to the device and back
  // as plain bytes, inside their metadata structs).
  Queue(const Queue&) = delete;
  Queue& operator=(const Queue&) = delete;

  void Init(length_t length) {
    if (alreadyInit_ && length == maxLen_) return;
    release();
    maxLen_ = length;
    queue_ = static_cast<T*>(allocDeviceArray(length, sizeof(T)));
    queueCurr_ = queueEnd_ = 0;
    devQueue_ = static_cast<Queue<T>*>(allocDeviceArray(1, sizeof(Queue<T>)));
    alreadyInit_ = true;
    SyncDeviceWithHost();
  }

  __device__ void enqueue(T t) {
    const length_t at = atomicAdd(&queueEnd_, 1);
    queue_[at] = t;
  }
  void enqueueFromHost(T t) {
    copyArrayHostToDevice(&t, queue_ + queueEnd_, 1, sizeof(T));
    ++queueEnd_;
  }

  T* getQueue() { return queue_; }
  __host__ __device__ length_t getQueueEnd() { return queueEnd_; }
  __host__ __device__ length_t getQueueCurr() { return queueCurr_; }
  void setQueueCurr(length_t curr) { queueCurr_ = curr; }
  void setQueueEnd(length_t end) { queueEnd_ = end; }
  void resetQueue() { queueCurr_ = queueEnd_ = 0; }
  length_t getActiveQueueSize() { return queueEnd_ - queueCurr_; }
  T* getQueueAtCurr() { return queue_ + queueCurr_; }
  T* getQueueAtEnd() { return queue_ + queueEnd_; }

  // Exchange the contents (array and indices) of two queues; ownership follows the arrays.
  static void swapQueues(Queue* q1, Queue* q2) {
    T* a = q1->queue_;
    const length_t c = q1->queueCurr_, e = q1->queueEnd_;
    q1->queue_ = q2->queue_;
    q1->queueCurr_ = q2->queueCurr_;
    q1->queueEnd_ = q2->queueEnd_;
    q2->queue_ = a;
    q2->queueCurr_ = c;
    q2->queueEnd_ = e;
  }

  // Release the arrays now (the destructor would otherwise do it); Init() may follow.
  void freeQueue() { release(); }

  Queue<T>* devPtr() { return devQueue_; }
  void SyncHostWithDevice() {
    Queue<T> tmp_bytes_only;  // receives the device copy's fields, then only the indices are kept
    copyArrayDeviceToHost(devQueue_, &tmp_bytes_only, 1, sizeof(Queue<T>));
    queueCurr_ = tmp_bytes_only.queueCurr_;
    queueEnd_ = tmp_bytes_only.queueEnd_;
    tmp_bytes_only.alreadyInit_ = false;  // the copy owns nothing
  }
  void SyncDeviceWithHost() { copyArrayHostToDevice(this, devQueue_, 1, sizeof(Queue<T>)); }

 private:
  void release() {
    if (!alreadyInit_) return;
    freeDeviceArray(queue_);
    freeDeviceArray(devQueue_);
    queue_ = nullptr;
    devQueue_ = nullptr;
    alreadyInit_ = false;
  }

  T* queue_ = nullptr;
  length_t queueCurr_ = 0;
  length_t queueEnd_ = 0;
  length_t maxLen_ = 0;
  bool alreadyInit_ = false;
  Queue<T>* devQueue_ = nullptr;
};

typedef Queue<vertexId_t> vertexQueue;

}  // namespace cuStingerAlgs

#endif
