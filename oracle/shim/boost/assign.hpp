/* TEST INFRASTRUCTURE ONLY: stand-in for boost::assign::map_list_of. */
#ifndef ORC_SHIM_ASSIGN_HPP
#define ORC_SHIM_ASSIGN_HPP
#include <map>
#include <string>
#include <utility>
#include <vector>
namespace boost { namespace assign {
template <class K, class V> class map_list {
    std::vector<std::pair<K, V>> items_;
public:
    map_list(const K &k, const V &v) { items_.emplace_back(k, v); }
    map_list &operator()(const K &k, const V &v) { items_.emplace_back(k, v); return *this; }
    template <class K2, class V2> operator std::map<K2, V2>() const
    {
        std::map<K2, V2> m;
        for (const auto &kv : items_) m.emplace(K2(kv.first), V2(kv.second));
        return m;
    }
};
template <class K, class V> map_list<const char *, V> map_list_of(const K &k, const V &v)
{
    return map_list<const char *, V>(k, v);
}
} }
#endif
