// Host worker threads shared by the library's parallel host stages
// (planning, lowering, ordering plans, trie building, descriptor filling,
// the halves of a batched run).  Creating threads per stage cost tens of
// microseconds per thread on every call; the workers here are created once
// and sleep between jobs.
#pragma once

#include <functional>

namespace gva {

// Runs fn(t) for every t in [0, n): the calling thread takes part, idle
// workers take the rest.  Returns when every call has returned.  Jobs may be
// submitted from several threads at once and from inside a job (the caller
// can always finish its own job alone, so nesting never waits on a busy
// worker).  fn must not throw.
void pool_run(unsigned n, const std::function<void(unsigned)>& fn);

// Threads a job can use at once: the workers plus the caller.
unsigned pool_width();

// Runs fn later on a background thread (in submission order); for work
// whose result nobody waits for, such as freeing the many small heap blocks
// of a finished batch's plans (milliseconds of free() calls that would
// otherwise sit on the caller's path).
void defer(std::function<void()> fn);

}  // namespace gva
