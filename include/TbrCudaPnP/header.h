// Drop-in for <TbrCudaPnP/header.h> (header.h:1-34), the one header the
// reference's evaluator includes: standard headers plus the estimator API.
#ifndef TBR_SHIM_HEADER_H
#define TBR_SHIM_HEADER_H

#include <algorithm>
#include <array>
#include <cerrno>
#include <cfenv>
#include <chrono>
#include <climits>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <TbrCudaPnP/ticktock.h>
#include <TbrCudaPnP/config.h>
#include <TbrCudaPnP/entry.h>
#include <TbrCudaPnP/camera.cuh>
#include <TbrCudaPnP/ba.cuh>

#endif
