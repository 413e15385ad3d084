// See gpu_btree.h.
#include "gpu_btree.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>

#include <cuda_runtime.h>

namespace eirene_b200 {

namespace {
void check(int rc, const char* what, int line) {
  if (rc != BT_OK) {
    std::printf("Error: %s:%d, code:%d, reason: %s\n", what, line, rc, bt_status_string(rc));
    std::exit(1);
  }
}
void check_cuda(cudaError_t e, const char* what, int line) {
  if (e != cudaSuccess) {
    std::printf("Error: %s:%d, code:%d, reason: %s\n", what, line, (int)e, cudaGetErrorString(e));
    std::exit(1);
  }
}
#define BT_CHECK(x) check((x), __FILE__, __LINE__)
#define BT_CUDA(x) check_cuda((x), __FILE__, __LINE__)
}  // namespace

BTree::BTree(int mode, bool learned, int device, uint64_t max_keys, uint64_t batch_size)
    : mode_(mode), learned_(learned), device_(device), max_keys_(max_keys), batch_size_(batch_size) {}

BTree::~BTree() {
  if (h_) bt_destroy(h_);
}

void BTree::prepareGPU() {
  bt_config c;
  BT_CHECK(bt_config_init(&c));
  c.max_keys = max_keys_;
  c.max_batch = batch_size_;
  c.device = device_;
  BT_CHECK(bt_create(&c, &h_));
}

// "R key" -> GET, "P key val" -> INSERT (value to the warehouse), "G lo hi" ->
// RANGE; lines that do not parse are skipped (src/input-helper.h:257-317)
void BTree::prepareInput(const std::string& fileName) {
  keys.clear();
  vals.clear();
  mission.clear();
  std::ifstream f(fileName);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    char type = 0;
    ss >> type;
    uint64_t k = 0, v = 0;
    if (type == 'R') {
      if (!(ss >> k)) continue;
      keys.push_back(k);
      mission.push_back(GET);
      vals.push_back(0);
    } else if (type == 'P') {
      if (!(ss >> k >> v)) continue;
      keys.push_back(k);
      mission.push_back(INSERT);
      vals.push_back(warehouse.size());
      warehouse.push_back(v);
    } else if (type == 'G') {
      if (!(ss >> k >> v)) continue;
      keys.push_back(k);
      mission.push_back(RANGE);
      vals.push_back(v);
    }
  }
}

// a file of bare keys with one mission (src/input-helper.h:201-255): INSERT
// stores the key itself as its value
void BTree::prepareInput(const std::string& fileName, Mission m) {
  keys.clear();
  vals.clear();
  mission.clear();
  std::ifstream f(fileName);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    uint64_t k = 0;
    if (!(ss >> k)) continue;
    keys.push_back(k);
    mission.push_back(m);
    if (m == INSERT) {
      vals.push_back(warehouse.size());
      warehouse.push_back(k);
    } else if (m == RANGE) {
      // "lo hi"; a line without an end ranges to the largest key
      // (the reference's INT_MAX, src/input-helper.h:105-116)
      uint64_t hi = 0;
      vals.push_back((ss >> hi) ? hi : ~0ull);
    } else {
      vals.push_back(0);
    }
  }
}

// batches of batch_size requests: H2D, one bt_execute_batch, D2H
// (src/gpu-stm-tree-v39/bpt-gpustm.cpp:67-132); device time of the batches
// summed as in the reference's "total gpu exec time"
void BTree::gpu_work() {
  const size_t n = keys.size();
  ans_vals.assign(n, 0);
  ans_status.assign(n, 0);
  uint64_t *dk = nullptr, *dv = nullptr, *dov = nullptr;
  uint8_t *dop = nullptr, *dos = nullptr;
  const size_t b = batch_size_;
  BT_CUDA(cudaMalloc(&dk, b * 8));
  BT_CUDA(cudaMalloc(&dv, b * 8));
  BT_CUDA(cudaMalloc(&dov, b * 8));
  BT_CUDA(cudaMalloc(&dop, b));
  BT_CUDA(cudaMalloc(&dos, b));
  cudaEvent_t e0, e1;
  BT_CUDA(cudaEventCreate(&e0));
  BT_CUDA(cudaEventCreate(&e1));
  float total_ms = 0;
  std::cout << "bucket size\t" << b << std::endl;
  std::cout << "total size\t" << n << std::endl;
  for (size_t s = 0; s < n; s += b) {
    const size_t m = std::min(b, n - s);
    BT_CUDA(cudaMemcpy(dk, keys.data() + s, m * 8, cudaMemcpyHostToDevice));
    BT_CUDA(cudaMemcpy(dv, vals.data() + s, m * 8, cudaMemcpyHostToDevice));
    BT_CUDA(cudaMemcpy(dop, mission.data() + s, m, cudaMemcpyHostToDevice));
    BT_CUDA(cudaEventRecord(e0));
    BT_CHECK(bt_execute_batch(h_, dk, dv, dop, dov, dos, m, mode_, nullptr));
    BT_CUDA(cudaEventRecord(e1));
    BT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    total_ms += ms;
    BT_CUDA(cudaMemcpy(ans_vals.data() + s, dov, m * 8, cudaMemcpyDeviceToHost));
    BT_CUDA(cudaMemcpy(ans_status.data() + s, dos, m, cudaMemcpyDeviceToHost));
  }
  gpu_seconds_ = total_ms / 1e3;
  std::cout << "total gpu exec time: " << gpu_seconds_ << std::endl;
  if (learned_) {
    BT_CHECK(bt_retrain(h_, nullptr));
    BT_CHECK(bt_set_descent(h_, BT_DESCENT_LEARNED));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dk);
  cudaFree(dv);
  cudaFree(dov);
  cudaFree(dop);
  cudaFree(dos);
}

// range queries keys[i] .. vals[i] (both included), batch_size at a time
void BTree::gpu_work_range() {
  const size_t n = keys.size();
  const size_t b = batch_size_;
  range_counts.assign(n, 0);
  range_keys.assign(n * range_max, 0);
  range_vals.assign(n * range_max, 0);
  uint64_t *dlo = nullptr, *dhi = nullptr, *dk = nullptr, *dv = nullptr;
  uint32_t* dc = nullptr;
  BT_CUDA(cudaMalloc(&dlo, b * 8));
  BT_CUDA(cudaMalloc(&dhi, b * 8));
  BT_CUDA(cudaMalloc(&dc, b * 4));
  BT_CUDA(cudaMalloc(&dk, b * range_max * 8 + 8));
  BT_CUDA(cudaMalloc(&dv, b * range_max * 8 + 8));
  cudaEvent_t e0, e1;
  BT_CUDA(cudaEventCreate(&e0));
  BT_CUDA(cudaEventCreate(&e1));
  float total_ms = 0;
  std::cout << "bucket size\t" << b << std::endl;
  std::cout << "total size\t" << n << std::endl;
  for (size_t s = 0; s < n; s += b) {
    const size_t m = std::min(b, n - s);
    BT_CUDA(cudaMemcpy(dlo, keys.data() + s, m * 8, cudaMemcpyHostToDevice));
    BT_CUDA(cudaMemcpy(dhi, vals.data() + s, m * 8, cudaMemcpyHostToDevice));
    BT_CUDA(cudaEventRecord(e0));
    BT_CHECK(bt_range_batch(h_, dlo, dhi, m, range_max, dk, dv, dc, nullptr));
    BT_CUDA(cudaEventRecord(e1));
    BT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    total_ms += ms;
    BT_CUDA(cudaMemcpy(range_counts.data() + s, dc, m * 4, cudaMemcpyDeviceToHost));
    BT_CUDA(cudaMemcpy(range_keys.data() + s * range_max, dk, m * range_max * 8, cudaMemcpyDeviceToHost));
    BT_CUDA(cudaMemcpy(range_vals.data() + s * range_max, dv, m * range_max * 8, cudaMemcpyDeviceToHost));
  }
  gpu_seconds_ = total_ms / 1e3;
  std::cout << "total gpu exec time: " << gpu_seconds_ << std::endl;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dlo);
  cudaFree(dhi);
  cudaFree(dc);
  cudaFree(dk);
  cudaFree(dv);
}

// per query: its bounds and full count, then its first range_max pairs (the
// stored value is a warehouse offset when the tree was loaded from P lines)
void BTree::test_range() {
  for (size_t i = 0; i < keys.size(); i++) {
    const uint32_t c = range_counts[i];
    std::cout << "range: " << keys[i] << " " << vals[i] << "\t count: " << c << "\n";
    const uint32_t shown = c < range_max ? c : range_max;
    for (uint32_t j = 0; j < shown; j++) {
      const uint64_t v = range_vals[i * range_max + j];
      std::cout << "  key: " << range_keys[i * range_max + j] << "\t ans: " << v;
      if (v < warehouse.size()) std::cout << "\t vals: " << warehouse[v];
      std::cout << "\n";
    }
  }
  std::cout.flush();
}

// one line per request; a found answer prints the warehouse offset and value
void BTree::test() {
  for (size_t i = 0; i < keys.size(); i++) {
    if (ans_status[i] == BT_ST_FOUND)
      std::cout << "key: " << keys[i] << "\t operator " << (int)mission[i] << "\t ans: " << ans_vals[i]
                << "\t vals: " << warehouse[ans_vals[i]] << "\n";
    else
      std::cout << "key: " << keys[i] << "\t operator " << (int)mission[i] << "\t ans: -1\n";
  }
  std::cout.flush();
}

}  // namespace eirene_b200
