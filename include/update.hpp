// update.hpp - batch update types of the cuStinger API subset (BatchUpdateData, BatchUpdate;
// cuStinger core, absent from the reference tree; used at tests/cct_upd.cpp:282-342,390-405 and
// by the streaming kernels, src/streaming_triangle_counting/cct_upd.cu:235-242,252,296-298,328-329).
//
// A BatchUpdateData holds `batchSize` directed entries (src[i], dst[i]) either in host memory
// (filled by the caller) or in device memory. BatchUpdate copies a host batch to the device;
// sortDeviceBUD() sorts it by (src, dst), builds the batch CSR offsets over src and flags
// repeated entries in indDuplicate; cuStinger::edgeInsertionsSorted additionally flags entries
// that were already in the graph. Self-loop entries are flagged as duplicates (the graph stays
// simple). Streaming triangle counting expects symmetric batches (both directions of every
// edge), as the reference driver builds them (tests/cct_upd.cpp:337-341).
#ifndef CUSTINGER_UPDATE_HPP_
#define CUSTINGER_UPDATE_HPP_

#include "cuStingerDefs.hpp"

class BatchUpdateData {
 public:
  BatchUpdateData(length_t batchSize, bool isHost, length_t nv = 0);
  ~BatchUpdateData();
  BatchUpdateData(const BatchUpdateData&) = delete;
  BatchUpdateData& operator=(const BatchUpdateData&) = delete;

  CUS_HD vertexId_t* getSrc() const { return src_; }
  CUS_HD vertexId_t* getDst() const { return dst_; }
  CUS_HD length_t* getBatchSize() const { return batchSize_; }
  CUS_HD length_t* getNumVertices() const { return numVertices_; }
  CUS_HD length_t* getIndDuplicate() const { return indDuplicate_; }
  CUS_HD length_t* getOffsets() const { return offsets_; }
  CUS_HD length_t* getvNumDuplicates() const { return vNumDuplicates_; }
  bool getisHost() const { return isHost_; }

  // Device copy of this object (device batches only), for kernels taking BatchUpdateData*.
  BatchUpdateData* devicePtr();

 private:
  vertexId_t* src_ = nullptr;
  vertexId_t* dst_ = nullptr;
  length_t* batchSize_ = nullptr;
  length_t* numVertices_ = nullptr;
  length_t* indDuplicate_ = nullptr;
  length_t* offsets_ = nullptr;
  length_t* vNumDuplicates_ = nullptr;
  bool isHost_ = true;
  length_t capacity_ = 0;
  length_t nv_ = 0;
  BatchUpdateData* d_self_ = nullptr;
  friend class BatchUpdate;
};

class BatchUpdate {
 public:
  explicit BatchUpdate(BatchUpdateData& hostBatch);
  ~BatchUpdate();
  BatchUpdate(const BatchUpdate&) = delete;
  BatchUpdate& operator=(const BatchUpdate&) = delete;

  BatchUpdateData* getHostBUD() { return host_; }
  BatchUpdateData* getDeviceBUD() { return dev_; }

  // Sort the device batch by (src, dst), build its CSR offsets, flag repeated entries.
  void sortDeviceBUD(const int blockdim);
  bool isSorted() const { return sorted_; }

 private:
  BatchUpdateData* host_;
  BatchUpdateData* dev_;
  bool sorted_ = false;
};

// Sort the batch on the device and check the result on the host, printing one line (the
// reference driver's sort test, tests/cct_upd.cpp:30,173).
void testSort(length_t nv, BatchUpdate& bu, const int blockdim);

#endif
