// Host-side tree plugin over the C ABI, mirroring the reference's plugin
// interface GPU_BTree (src/tree.h:28-43): same member names, the same text
// request format (src/input-helper.h:161-163: "R key", "P key val",
// "G start end"), the same value "warehouse" (an INSERT stores its value in a
// host vector and the tree holds the value's offset, src/input-helper.h:
// 289-299), and the same answer print of test() (src/input-helper.h:327-340).
// Like the reference's CUDA_ERROR_HANDLER (src/cuda_utils.h:3-12) an error
// prints the reason and exits.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "eirene_b200.h"

namespace eirene_b200 {

// op codes as in src/input-helper.h:14-17
enum Mission : uint8_t { INSERT = 0, GET = 1, DELETE = 2, RANGE = 3 };

class GPU_BTree {
 public:
  virtual ~GPU_BTree() {}
  virtual void prepareGPU() = 0;
  virtual void prepareInput(const std::string& fileName) = 0;
  virtual void prepareInput(const std::string& fileName, Mission m) { (void)fileName; (void)m; }
  virtual void gpu_work() = 0;
  virtual void gpu_work_sp() {}
  virtual void gpu_work_range() {}
  virtual void test() = 0;
  virtual void test_range() {}
};

// mode: BT_MODE_STM (the v39 meaning), BT_MODE_SORTED (v38), optionally
// | BT_MODE_MERGE_ENGINE; learned selects the learned descent after loading.
class BTree : public GPU_BTree {
 public:
  explicit BTree(int mode, bool learned = false, int device = 0, uint64_t max_keys = 1ull << 27,
                 uint64_t batch_size = 1310720);
  ~BTree() override;
  void prepareGPU() override;
  void prepareInput(const std::string& fileName) override;
  void prepareInput(const std::string& fileName, Mission m) override;
  void gpu_work() override;
  void gpu_work_sp() override { gpu_work(); }
  // range files (-r): the reference declares these members but leaves them
  // empty in every version (src/tree.h:37-39); here each "lo [hi]" query runs
  // through bt_range_batch and test_range prints its count and first pairs
  void gpu_work_range() override;
  void test_range() override;
  void test() override;
  double last_gpu_seconds() const { return gpu_seconds_; }
  bt_handle* handle() const { return h_; }

  // requests of the current input (public for drivers and tests)
  std::vector<uint64_t> keys, vals;  // vals: warehouse offsets for INSERT
  std::vector<uint8_t> mission;
  std::vector<uint64_t> warehouse;  // true values
  std::vector<uint64_t> ans_vals;
  std::vector<uint8_t> ans_status;
  // range answers: full count per query and its first range_max pairs
  uint32_t range_max = 16;
  std::vector<uint32_t> range_counts;
  std::vector<uint64_t> range_keys, range_vals;

 private:
  int mode_;
  bool learned_;
  int device_;
  uint64_t max_keys_, batch_size_;
  bt_handle* h_ = nullptr;
  double gpu_seconds_ = 0;
};

}  // namespace eirene_b200
