/* TEST INFRASTRUCTURE ONLY: minimal stand-in for boost::format supporting the
 * "%|0N|" directives the reference uses in file names. */
#ifndef ORC_SHIM_FORMAT_HPP
#define ORC_SHIM_FORMAT_HPP
#include <iomanip>
#include <ostream>
#include <sstream>
#include <string>
namespace boost {
class format {
    std::string fmt_, out_;
    std::size_t pos_ = 0;
    void flush_literal()
    {
        while (pos_ < fmt_.size()) {
            if (fmt_[pos_] == '%' && pos_ + 1 < fmt_.size() && fmt_[pos_ + 1] == '|') return;
            out_ += fmt_[pos_++];
        }
    }
public:
    explicit format(const std::string &f) : fmt_(f) { flush_literal(); }
    template <class T> format &operator%(const T &v)
    {
        if (pos_ >= fmt_.size()) return *this;
        std::size_t end = fmt_.find('|', pos_ + 2);
        std::string spec = fmt_.substr(pos_ + 2, end - pos_ - 2);
        std::ostringstream os;
        if (!spec.empty() && spec[0] == '0') os << std::setfill('0');
        if (!spec.empty()) os << std::setw(std::stoi(spec));
        os << v;
        out_ += os.str();
        pos_ = end + 1;
        flush_literal();
        return *this;
    }
    std::string str() const { return out_; }
    friend std::ostream &operator<<(std::ostream &o, const format &f) { return o << f.out_; }
};
}
#endif
