/* matplotlib-cpp stand-in used ONLY to compile the reference's sources for
 * parity checks: plotting is a display aid (utils/globals.cpp:17-129) and is
 * compiled to no-ops.  Also supplies <algorithm>, which
 * simulated_pulsar/simulated_complex_signal.cpp uses without including. */
#ifndef MSOSM_REF_SHIM_MATPLOTLIBCPP_H
#define MSOSM_REF_SHIM_MATPLOTLIBCPP_H
#include <algorithm>
#include <string>
#include <vector>
namespace matplotlibcpp {
template <typename T> inline bool plot(const std::vector<T> &) { return true; }
template <typename T, typename U> inline bool plot(const std::vector<T> &, const std::vector<U> &) { return true; }
inline void show() {}
namespace detail {
struct _interpreter {
    static void kill() {}
};
} // namespace detail
} // namespace matplotlibcpp
#endif
