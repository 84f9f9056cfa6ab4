// Wall-clock stopwatch with the interface the diffusion3d plugin surface
// uses (StopwatchStart / StopwatchStop returning seconds as float; the
// reference's is src/common/stopwatch.h:17-45), on a monotonic clock.
#ifndef BENCHMARKS_B200_MIRROR_STOPWATCH_H_
#define BENCHMARKS_B200_MIRROR_STOPWATCH_H_

#include <time.h>

typedef struct {
  struct timespec ts;
} Stopwatch;

static inline void StopwatchStart(Stopwatch* w) {
  clock_gettime(CLOCK_MONOTONIC, &w->ts);
}

static inline float StopwatchStop(Stopwatch* w) {
  struct timespec now;
  clock_gettime(CLOCK_MONOTONIC, &now);
  return (float)((double)(now.tv_sec - w->ts.tv_sec) +
                 1.0e-9 * (double)(now.tv_nsec - w->ts.tv_nsec));
}

#endif  // BENCHMARKS_B200_MIRROR_STOPWATCH_H_
