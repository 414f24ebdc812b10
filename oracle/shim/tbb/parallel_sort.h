// Stand-in for TBB's parallel_sort, which this image lacks; the reference's
// CPU sorter (src/sort/parallel_sorter.cpp:9,28) only needs an ordering.
#pragma once
#include <algorithm>
namespace tbb {
template <class It> void parallel_sort(It first, It last) { std::sort(first, last); }
}  // namespace tbb
