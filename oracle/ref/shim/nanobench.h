// Test-infrastructure shim: nanobench is not installed here; the reference's
// benchmark bodies compile against this no-op stand-in and are never run.
#pragma once
#include <ostream>
namespace ankerl::nanobench {
namespace templates {
    inline const char* json() { return ""; }
}
class Bench {
public:
    Bench& title(const char*) { return *this; }
    Bench& minEpochIterations(unsigned long) { return *this; }
    template <typename F> Bench& run(const char*, F&&) { return *this; }
    template <typename T> void render(T, std::ostream&) { }
};
}
