// Stand-in for MSVC's <ppl.h> used by the YMRT reference (BVH builders, scene
// module). Runs the loop body sequentially, in index order: the reference's
// builders produce the same tree either way, and a fixed order keeps the
// oracle deterministic. Test infrastructure only.
#pragma once
namespace concurrency {
template <typename Index, typename Function>
inline void parallel_for(Index first, Index last, const Function& body) {
  for (Index i = first; i < last; ++i) body(i);
}
}  // namespace concurrency
