// Stand-in for the reference's main/src/Logger.cpp (which needs boost::iostreams):
// the oracle build logs nothing, so every request goes to a stream without a buffer.  Such a
// stream is in the bad state, so formatted output returns at once without touching a locale;
// it is built on first use, after every static initialiser of the library has run.
#include <ostream>

namespace logger {
  namespace {
    int level = 0;
  } // namespace
  std::ostream& logger(int)
  {
    static std::ostream null_stream(nullptr);
    return null_stream;
  }
  int verbosity() { return level; }
  void setVerbosity(int l) { level = l; }
} // namespace logger
