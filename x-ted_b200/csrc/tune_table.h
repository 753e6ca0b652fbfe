// tune_table.h -- granularity per tree-size bucket, written by
// x-ted_b200/xted/autotune.py (do not edit by hand; rerun the tuner).
//
// Row k applies to trees with fewer than max_n nodes (the last row to all
// larger ones): the row-run length of the tree as a row tree, and the widest
// narrow (one warp) and half-block chunks of the tree as a column tree.
// sizes [50, 128), 8192 pairs: best 70.45 ms (run_rows 32, narrow 128, half -1), untuned default 71.48 ms
// sizes [128, 256), 4096 pairs: best 82.05 ms (run_rows 128, narrow 256, half 384), untuned default 83.43 ms
// sizes [256, 512), 2048 pairs: best 83.88 ms (run_rows 64, narrow 256, half 512), untuned default 83.88 ms
// sizes [512, 1024), 1024 pairs: best 121.64 ms (run_rows 128, narrow 128, half 512), untuned default 127.70 ms
// sizes [1024, 2048), 384 pairs: best 162.51 ms (run_rows 128, narrow 128, half 512), untuned default 167.17 ms
// sizes [2048, 4096), 96 pairs: best 1756.62 ms (run_rows 64, narrow 128, half 384), untuned default 1875.39 ms
// 24 candidates per bucket, 207 s on a B200
#pragma once

#include "xted_internal.h"

static const XTuneRow kTuneTable[] = {
    {128, 32, 128, -1},
    {256, 128, 256, 384},
    {512, 64, 256, 512},
    {1024, 128, 128, 512},
    {2048, 128, 128, 512},
    {1 << 30, 64, 128, 384},
};
static const int kTuneRows = (int)(sizeof(kTuneTable) / sizeof(kTuneTable[0]));
