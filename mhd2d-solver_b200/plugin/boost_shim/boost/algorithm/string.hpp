// Project-written stand-in for boost::replace_all (Boost.StringAlgo), the
// one string algorithm the reference's output naming uses
// (file_access.cpp:233-246, 1234-1236, 1360-1362): every non-overlapping
// occurrence of `from`, scanned left to right, is replaced by `to`.
#ifndef MHD2D_B200_SHIM_ALGORITHM_STRING_HPP
#define MHD2D_B200_SHIM_ALGORITHM_STRING_HPP

#include <string>

namespace boost {
namespace algorithm {

inline void replace_all(std::string& input, const std::string& from, const std::string& to) {
  if (from.empty()) return;
  std::string out;
  size_t pos = 0;
  for (;;) {
    const size_t hit = input.find(from, pos);
    if (hit == std::string::npos) break;
    out.append(input, pos, hit - pos);
    out.append(to);
    pos = hit + from.size();
  }
  out.append(input, pos, std::string::npos);
  input.swap(out);
}

}  // namespace algorithm

using algorithm::replace_all;

}  // namespace boost

#endif
