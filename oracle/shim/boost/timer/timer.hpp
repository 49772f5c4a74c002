/* TEST INFRASTRUCTURE ONLY: stand-in for boost::timer::cpu_timer (wall clock). */
#ifndef ORC_SHIM_TIMER_HPP
#define ORC_SHIM_TIMER_HPP
#include <chrono>
namespace boost { namespace timer {
struct cpu_times { long long wall, user, system; };
class cpu_timer {
    std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();
public:
    cpu_times elapsed() const
    {
        auto d = std::chrono::steady_clock::now() - t0_;
        return cpu_times{(long long)std::chrono::duration_cast<std::chrono::nanoseconds>(d).count(), 0, 0};
    }
};
} }
#endif
