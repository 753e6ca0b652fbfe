// tune_table.h -- granularity per tree-size bucket, written by
// x-ted_b200/xted/autotune.py (do not edit by hand; rerun the tuner).
//
// Row k applies to trees with fewer than max_n nodes (the last row to all
// larger ones): the row-run length of the tree as a row tree, and the widest
// narrow (one warp) and half-block chunks of the tree as a column tree.
// sizes [50, 128), 8192 pairs: best 64.77 ms (run_rows 128, narrow 256, half 768), untuned default 65.02 ms
// sizes [128, 256), 4096 pairs: best 66.10 ms (run_rows 128, narrow 256, half 768), untuned default 68.79 ms
// sizes [256, 512), 2048 pairs: best 60.72 ms (run_rows 128, narrow 256, half 1024), untuned default 63.33 ms
// sizes [512, 1024), 1024 pairs: best 97.99 ms (run_rows 128, narrow 256, half 512), untuned default 100.95 ms
// sizes [1024, 2048), 384 pairs: best 146.40 ms (run_rows 128, narrow 128, half 512), untuned default 154.11 ms
// sizes [2048, 4096), 96 pairs: best 275.13 ms (run_rows 128, narrow 128, half 512), untuned default 321.96 ms
// 40 candidates per bucket, 128 s on a B200
#pragma once

#include "xted_internal.h"

static const XTuneRow kTuneTable[] = {
    {128, 128, 256, 768},
    {256, 128, 256, 768},
    {512, 128, 256, 1024},
    {1024, 128, 256, 512},
    {2048, 128, 128, 512},
    {1 << 30, 128, 128, 512},
};
static const int kTuneRows = (int)(sizeof(kTuneTable) / sizeof(kTuneTable[0]));
