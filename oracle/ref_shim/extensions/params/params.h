// A restatement, written for this repository, of the parameter dictionary
// interface that the reference takes from argsparser v0.0.9's
// extensions/params (not available here). It provides only what the
// reference's sources call (src/param/params.h, xamg_params_details.h,
// api/c/xamg_c_api.cpp, solvers/*, hypre/*), with the behaviour those call
// sites imply: named lists of typed key/value pairs, a family key, family and
// dictionary defaults supplied by the details class, per-level overrides
// written "value@levA-B", and checks against the expected-parameter table.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref): it lets the reference's solve phase
// compile and run on one rank as a parity pin for the CPU oracle.
//
// The reference includes this file inside namespace XAMG, so it includes no
// headers itself: the translation unit that includes the reference's sources
// includes <map>, <string>, <vector>, <sstream>, <cstdio>, <cstdlib>,
// <stdexcept> and <utility> first.

namespace params {

namespace value {
enum type_t { S, I, F };
}

struct expected_param {
    value::type_t type;
    bool flag;  // second column of the table (not needed by the checks here)
    std::vector<std::string> families;
    std::vector<std::string> minmax;
    std::vector<std::string> allowed;
};
typedef std::map<std::string, expected_param> expected_params_t;

namespace detail {
inline std::string to_text(const std::string &v) { return v; }
inline std::string to_text(const char *v) { return v; }
inline std::string to_text(float v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.9g", (double)v);
    return b;
}
inline std::string to_text(double v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%.17g", v);
    return b;
}
template <typename T>
inline std::string to_text(T v) {
    return std::to_string((long long)v);
}
template <typename T>
inline T from_text(const std::string &s, T *) {
    return (T)std::strtoll(s.c_str(), nullptr, 10);
}
inline float from_text(const std::string &s, float *) { return std::strtof(s.c_str(), nullptr); }
inline double from_text(const std::string &s, double *) { return std::strtod(s.c_str(), nullptr); }
inline std::string from_text(const std::string &s, std::string *) { return s; }
inline bool from_text(const std::string &s, bool *) { return std::strtoll(s.c_str(), nullptr, 10); }
inline void fail(const std::string &what) { throw std::runtime_error("params: " + what); }
}  // namespace detail

template <class D>
class list {
  public:
    std::map<std::string, std::string> kv;

    bool find(const std::string &key) const { return kv.count(key) > 0; }
    template <typename T>
    T get_value(const std::string &key) const {
        auto it = kv.find(key);
        if (it == kv.end()) detail::fail("no value for key '" + key + "'");
        return detail::from_text(it->second, (T *)nullptr);
    }
    template <typename T>
    void get_value(const std::string &key, T &out) const {
        out = get_value<T>(key);
    }
    template <typename T>
    void add_value(const std::string &key, const T &v) {
        check(key, detail::to_text(v));
        kv[key] = detail::to_text(v);
    }
    template <typename T>
    void set_value_if_missing(const std::string &key, const T &v) {
        if (!find(key)) add_value(key, v);
    }
    template <typename T>
    void change_value(const std::string &key, const T &v) {
        if (!find(key)) detail::fail("change_value of absent key '" + key + "'");
        add_value(key, v);
    }
    void set_text(const std::string &key, const std::string &v) {
        check(key, v);
        kv[key] = v;
    }
    // the other list's entries replace or add to this one's
    void override_params(const list &other) {
        for (auto &e : other.kv) kv[e.first] = e.second;
    }
    void erase() { kv.clear(); }

    // a key must be in the expected table, and a numeric value within its
    // min/max and allowed set
    static void check(const std::string &key, const std::string &text) {
        const expected_params_t &t = D::get_expected_params();
        auto it = t.find(key);
        if (it == t.end()) detail::fail("unknown key '" + key + "'");
        const expected_param &e = it->second;
        if (e.type == value::S) return;
        const double x = std::strtod(text.c_str(), nullptr);
        if (e.minmax.size() == 2) {
            if (e.minmax[0] != "-inf" && x < std::strtod(e.minmax[0].c_str(), nullptr))
                detail::fail("'" + key + "' = " + text + " below its minimum");
            if (e.minmax[1] != "inf" && x > std::strtod(e.minmax[1].c_str(), nullptr))
                detail::fail("'" + key + "' = " + text + " above its maximum");
        }
        if (!e.allowed.empty()) {
            bool ok = false;
            for (auto &a : e.allowed) ok = ok || (x == std::strtod(a.c_str(), nullptr));
            if (!ok) detail::fail("'" + key + "' = " + text + " not an allowed value");
        }
    }

    static void print_line_delimiter() { std::printf("%s\n", std::string(64, '-').c_str()); }
    static void print_header(const std::string &h, int = 1) { std::printf("%s\n", h.c_str()); }
    void print(const std::string &title) const {
        std::printf("[%s]\n", title.c_str());
        for (auto &e : kv) std::printf("  %s = %s\n", e.first.c_str(), e.second.c_str());
    }
};

template <class D>
class dictionary {
  public:
    std::map<std::string, list<D>> lists;
    // list name -> level -> key -> value text
    std::map<std::string, std::map<int, std::map<std::string, std::string>>> overrides;

    bool find(const std::string &name) const { return lists.count(name) > 0; }

    // conds: (key, value) pairs, any of which selects a list
    template <typename T>
    bool find_if(const std::vector<std::pair<std::string, T>> &conds) const {
        for (auto &l : lists)
            if (matches(l.second, conds)) return true;
        return false;
    }
    template <typename T>
    const list<D> &get_if(const std::vector<std::pair<std::string, T>> &conds) const {
        for (auto &l : lists)
            if (matches(l.second, conds)) return l.second;
        detail::fail("no list matches");
        return lists.begin()->second;
    }
    template <typename T>
    list<D> &get_if(const std::vector<std::pair<std::string, T>> &conds, std::string &name) {
        for (auto &l : lists)
            if (matches(l.second, conds)) {
                name = l.first;
                return l.second;
            }
        detail::fail("no list matches");
        return lists.begin()->second;
    }
    template <typename T>
    const list<D> &get_if(const std::vector<std::pair<std::string, T>> &conds, std::string &name) const {
        for (auto &l : lists)
            if (matches(l.second, conds)) {
                name = l.first;
                return l.second;
            }
        detail::fail("no list matches");
        return lists.begin()->second;
    }

    list<D> &get(const std::string &name) {
        auto it = lists.find(name);
        if (it == lists.end()) detail::fail("no list '" + name + "'");
        return it->second;
    }
    const list<D> &get(const std::string &name) const {
        auto it = lists.find(name);
        if (it == lists.end()) detail::fail("no list '" + name + "'");
        return it->second;
    }
    // the list with the overrides of level lev applied
    list<D> get(const std::string &name, int lev) const {
        list<D> out;
        auto it = lists.find(name);
        if (it != lists.end()) out = it->second;
        auto o = overrides.find(name);
        if (o != overrides.end()) {
            auto l = o->second.find(lev);
            if (l != o->second.end())
                for (auto &e : l->second) out.kv[e.first] = e.second;
        }
        return out;
    }

    void add(const std::string &name, const list<D> &l) {
        for (auto &e : l.kv) lists[name].set_text(e.first, e.second);
    }
    void add(const std::string &name, const std::pair<std::string, std::string> &kv) {
        lists[name].set_text(kv.first, kv.second);
    }
    template <typename T>
    void change_value(const std::string &name, const std::string &key, const T &v) {
        get(name).change_value(key, v);
    }
    template <typename T>
    void forced_change_value(const std::string &name, const std::string &key, const T &v) {
        lists[name].add_value(key, v);
    }
    // "value@levA-B" (or "value@levA"), comma-separated specs
    void add_override(const std::string &name, const std::map<std::string, std::string> &ov) {
        for (auto &e : ov) {
            std::stringstream ss(e.second);
            std::string spec;
            while (std::getline(ss, spec, ',')) {
                const size_t at = spec.find("@lev");
                if (at == std::string::npos) detail::fail("override '" + spec + "'");
                const std::string val = spec.substr(0, at), range = spec.substr(at + 4);
                const size_t dash = range.find('-');
                const int a = std::atoi(range.substr(0, dash).c_str());
                const int b = dash == std::string::npos ? a : std::atoi(range.substr(dash + 1).c_str());
                list<D>::check(e.first, val);
                for (int l = a; l <= b; ++l) overrides[name][l][e.first] = val;
            }
        }
    }
    void set_defaults() {
        D::set_dictionary_defaults(*this);
        for (auto &l : lists)
            D::set_family_defaults(l.second, l.second.template get_value<std::string>(
                                                 D::get_family_key()),
                                   l.first);
    }
    void print() const { D::print_table(*this); }
    void print_list(const std::string &name, const std::string &title) const {
        auto it = lists.find(name);
        if (it != lists.end()) it->second.print(title);
    }

  private:
    template <typename T>
    static bool matches(const list<D> &l, const std::vector<std::pair<std::string, T>> &conds) {
        for (auto &c : conds)
            if (l.find(c.first) && l.template get_value<T>(c.first) == c.second) return true;
        return false;
    }
};

}  // namespace params
