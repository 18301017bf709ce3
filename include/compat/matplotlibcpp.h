// matplotlibcpp.h -- headless stand-in for matplotlib-cpp, which the
// reference's drivers include for display only (utils/include/globals.h).
// The namespace exists so that `namespace plt = matplotlibcpp;` compiles;
// plotting goes through the helpers of the compatibility globals.h.
#pragma once

namespace matplotlibcpp {
inline void show() {}
}  // namespace matplotlibcpp
