#pragma once
// Stand-in for the LHCb ODIN event header class (LHCb stack, absent here).  The reference's
// MDF transpose only asks it for a run and an event number when it meets an ODIN bank; those
// numbers never reach the VELO slice, so this class reads them from the first words of the bank
// without following the real ODIN layout.
#include <cstdint>
#include <gsl/gsl>

namespace LHCb {
  class ODIN {
  public:
    ODIN() = default;
    explicit ODIN(gsl::span<unsigned const> data)
    {
      if (data.size() > 0) m_run = data[0];
      if (data.size() > 1) m_event = data[1];
    }
    template<int VERSION>
    static ODIN from_version(gsl::span<unsigned const> data)
    {
      return ODIN(data);
    }
    unsigned runNumber() const { return m_run; }
    std::uint64_t eventNumber() const { return m_event; }

  private:
    unsigned m_run = 0;
    std::uint64_t m_event = 0;
  };
} // namespace LHCb
