// Stand-in for the reference's main/src/Logger.cpp (which needs boost::iostreams):
// the oracle build logs nothing, so every request goes to a discarding stream.
#include <ostream>
#include <streambuf>

namespace logger {
  namespace {
    struct NullBuffer : std::streambuf {
      int overflow(int c) override { return c; }
    };
    NullBuffer null_buffer;
    std::ostream null_stream(&null_buffer);
    int level = 0;
  } // namespace
  std::ostream& logger(int) { return null_stream; }
  int verbosity() { return level; }
  void setVerbosity(int l) { level = l; }
} // namespace logger
