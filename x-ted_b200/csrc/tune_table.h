// tune_table.h -- granularity per tree-size bucket, written by
// x-ted_b200/xted/autotune.py (do not edit by hand; rerun the tuner).
//
// Row k applies to trees with fewer than max_n nodes (the last row to all
// larger ones): the row-run length of the tree as a row tree, and the widest
// narrow (one warp) and half-block chunks of the tree as a column tree.
// sizes [50, 128), 8192 pairs: best 65.28 ms (run_rows 64, narrow 128, half -1), untuned default 65.35 ms
// sizes [128, 256), 4096 pairs: best 66.28 ms (run_rows 128, narrow 256, half -1), untuned default 68.75 ms
// sizes [256, 512), 2048 pairs: best 60.73 ms (run_rows 128, narrow 256, half 1024), untuned default 63.15 ms
// sizes [512, 1024), 1024 pairs: best 97.96 ms (run_rows 128, narrow 256, half 512), untuned default 100.79 ms
// sizes [1024, 2048), 384 pairs: best 146.34 ms (run_rows 128, narrow 128, half 512), untuned default 148.38 ms
// sizes [2048, 4096), 96 pairs: best 269.09 ms (run_rows 128, narrow 128, half 512), untuned default 323.79 ms
// mixed batches of [1024, 2048, 4096] pairs: [98.4, 126.44, 232.85] ms with the previous table, [98.4, 126.44, 232.85] ms with this one; rows taken from this run: [] (the others kept)
// 40 candidates per bucket, 131 s on a B200
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
