/* TEST INFRASTRUCTURE ONLY: stand-in for boost::alignment::aligned_alloc. */
#ifndef ORC_SHIM_ALIGNED_ALLOC_HPP
#define ORC_SHIM_ALIGNED_ALLOC_HPP
#include <cstdlib>
namespace boost { namespace alignment {
inline void *aligned_alloc(std::size_t a, std::size_t n)
{
    void *p = nullptr;
    if (posix_memalign(&p, a < sizeof(void *) ? sizeof(void *) : a, n ? n : a) != 0) return nullptr;
    return p;
}
inline void aligned_free(void *p) { std::free(p); }
} }
#endif
