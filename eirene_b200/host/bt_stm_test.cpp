// Command-line driver with the reference's options (src/main.cpp:57-109):
//   bt_stm_test -v<version> [-t] -i <requests> [-i <requests> ...]
// -v 39: warp STM batches (v39 meaning); -v 38: sort-merged batches (v38
// meaning); -v 40: sort-merged with the segmented leaf merge; -v 41: as 40
// with the learned descent after the first file.  -t prints the answers of
// the following files; -i runs a file of R/P/G lines; -s is a synonym of -i;
// -r runs a file of range queries, one "lo [hi]" per line (src/main.cpp:30-34).
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>

#include "gpu_btree.h"

int main(int argc, char* argv[]) {
  std::unique_ptr<eirene_b200::GPU_BTree> tree;
  bool test_flag = false;
  int opt;
  opterr = 0;
  while ((opt = getopt(argc, argv, "ts:i:r:v:")) != -1) {
    switch (opt) {
      case 't':
        test_flag = !test_flag;
        break;
      case 'v': {
        const int v = std::atoi(optarg);
        int mode = -1;
        bool learned = false;
        if (v == 39) mode = BT_MODE_STM;
        else if (v == 38) mode = BT_MODE_SORTED;
        else if (v == 40) mode = BT_MODE_SORTED | BT_MODE_MERGE_ENGINE;
        else if (v == 41) {
          mode = BT_MODE_SORTED | BT_MODE_MERGE_ENGINE;
          learned = true;
        }
        if (mode < 0) {
          std::fprintf(stderr, "unknown version %d (use 38, 39, 40 or 41)\n", v);
          return 2;
        }
        tree.reset(new eirene_b200::BTree(mode, learned));
        tree->prepareGPU();
        break;
      }
      case 'i':
      case 's':
        if (!tree) {
          std::fprintf(stderr, "-v must come first\n");
          return 2;
        }
        tree->prepareInput(optarg);
        tree->gpu_work();
        if (test_flag) tree->test();
        break;
      case 'r':
        if (!tree) {
          std::fprintf(stderr, "-v must come first\n");
          return 2;
        }
        tree->prepareInput(optarg, eirene_b200::RANGE);
        tree->gpu_work_range();
        if (test_flag) tree->test_range();
        break;
      default:
        std::fprintf(stderr, "usage: %s -v{38,39,40,41} [-t] -i file [-i file ...] [-r file]\n", argv[0]);
        return 2;
    }
  }
  if (!tree) {
    std::fprintf(stderr, "usage: %s -v{38,39,40,41} [-t] -i file [-i file ...]\n", argv[0]);
    return 2;
  }
  return 0;
}
