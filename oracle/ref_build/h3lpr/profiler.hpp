// Minimal stand-in for the h3lpr helper library's profiler.hpp: the
// Profiler type the reference passes around and the m_prof* macros it
// calls, as no-ops (the oracle build times solves from outside).  Test
// infrastructure of the oracle only.
#pragma once
#include <string>

namespace H3LPR {
class Profiler {
   public:
    Profiler() = default;
    explicit Profiler(const std::string& name) : name_(name) {}
    const std::string& name() const { return name_; }

   private:
    std::string name_;
};
}  // namespace H3LPR

#define m_profStart(prof, name) ((void)(prof), (void)(name))
#define m_profStop(prof, name) ((void)(prof), (void)(name))
#define m_profInitLeave(prof, name) ((void)(prof), (void)(name))
#define m_profDisp(prof) ((void)(prof))
