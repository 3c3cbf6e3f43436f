// Drop-in for <TbrCudaPnP/ticktock.h>: wall-clock helpers the evaluator's
// headers pull in (seconds / milliseconds since TICK).
#ifndef TBR_SHIM_TICKTOCK_H
#define TBR_SHIM_TICKTOCK_H

#include <chrono>
#include <iostream>

#define TICK(x) auto bench_##x = std::chrono::steady_clock::now();
#define TOCK(x)                                                                                        \
    std::cout << #x " time: "                                                                          \
              << std::chrono::duration<double>(std::chrono::steady_clock::now() - bench_##x).count()  \
              << " s" << std::endl;
#define TICK_MS(x) auto bench_##x = std::chrono::steady_clock::now();
#define TOCK_MS(x)                                                                                           \
    std::cout << #x " time: "                                                                                \
              << std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - bench_##x).count() \
              << " ms" << std::endl;

#endif
