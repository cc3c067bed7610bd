// TEST INFRASTRUCTURE: a stand-in for the part of the yaml-cpp API that the
// reference's input parser (Code/input.cpp) uses, so that the reference's own
// driver (Code/main.cpp) can be built in place against this library's backend
// shim where yaml-cpp is not installed.  Own implementation of a small YAML
// subset: block maps and block sequences by indentation, flow sequences
// [a, b, [c, d]] and flow maps {K: v}, plain and quoted scalars, # comments.
// Node API: operator bool (defined), operator[] by key or index, as<T>(),
// IsSequence/IsMap/IsScalar/IsNull/IsDefined, size(), iteration (map entries
// as .first/.second, sequence items as nodes), Node(NodeType::Sequence),
// LoadFile, Load, Exception.
#pragma once

#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace YAML {

struct Exception : std::runtime_error {
    explicit Exception(const std::string& m) : std::runtime_error(m) {}
};
struct BadFile : Exception {
    explicit BadFile(const std::string& f) : Exception("bad file: " + f) {}
};
struct ParserException : Exception {
    ParserException(int line, const std::string& m) : Exception("yaml line " + std::to_string(line) + ": " + m) {}
};
struct TypedBadConversion : Exception {
    explicit TypedBadConversion(const std::string& v) : Exception("bad conversion of '" + v + "'") {}
};

struct NodeType {
    enum value { Undefined, Null, Scalar, Sequence, Map };
};

class Node;

namespace detail {
struct Data {
    NodeType::value type = NodeType::Null;
    std::string scalar;
    std::vector<Node> seq;
    std::vector<std::pair<Node, Node>> map;
};
}  // namespace detail

class Node;

struct IterValue;

class Node {
public:
    Node() : d_(std::make_shared<detail::Data>()) {}
    explicit Node(NodeType::value t) : d_(std::make_shared<detail::Data>()) { d_->type = t; }
    explicit Node(const std::string& scalar) : d_(std::make_shared<detail::Data>())
    {
        d_->type = NodeType::Scalar;
        d_->scalar = scalar;
    }
    static Node undefined()
    {
        Node n;
        n.d_->type = NodeType::Undefined;
        return n;
    }

    NodeType::value Type() const { return d_->type; }
    bool IsDefined() const { return d_->type != NodeType::Undefined; }
    bool IsNull() const { return d_->type == NodeType::Null; }
    bool IsScalar() const { return d_->type == NodeType::Scalar; }
    bool IsSequence() const { return d_->type == NodeType::Sequence; }
    bool IsMap() const { return d_->type == NodeType::Map; }
    explicit operator bool() const { return IsDefined(); }
    bool operator!() const { return !IsDefined(); }

    std::size_t size() const
    {
        if (IsSequence()) return d_->seq.size();
        if (IsMap()) return d_->map.size();
        return 0;
    }

    Node operator[](const std::string& key) const
    {
        if (IsMap())
            for (const auto& kv : d_->map)
                if (kv.first.d_->scalar == key) return kv.second;
        return undefined();
    }
    Node operator[](const char* key) const { return (*this)[std::string(key)]; }
    Node operator[](std::size_t i) const
    {
        if (IsSequence() && i < d_->seq.size()) return d_->seq[i];
        return undefined();
    }
    Node operator[](int i) const { return i < 0 ? undefined() : (*this)[(std::size_t)i]; }

    template <class T>
    T as() const;

    // building (parser)
    void push_back(const Node& n) { d_->seq.push_back(n); }
    void add(const Node& k, const Node& v) { d_->map.emplace_back(k, v); }
    const std::string& scalar() const { return d_->scalar; }

    class const_iterator;
    const_iterator begin() const;
    const_iterator end() const;

private:
    std::shared_ptr<detail::Data> d_;
    friend class const_iterator;
};

// What iteration yields: a map entry (first = key, second = value) or a
// sequence item (the node itself; first and second undefined).
struct IterValue : Node {
    Node first, second;
    IterValue(const Node& self, const Node& f, const Node& s) : Node(self), first(f), second(s) {}
};

class Node::const_iterator {
public:
    const_iterator(const Node* n, std::size_t i) : n_(n), i_(i) {}
    IterValue operator*() const
    {
        if (n_->IsMap()) {
            const auto& kv = n_->d_->map[i_];
            return IterValue(kv.second, kv.first, kv.second);
        }
        return IterValue(n_->d_->seq[i_], Node::undefined(), Node::undefined());
    }
    const_iterator& operator++()
    {
        ++i_;
        return *this;
    }
    bool operator!=(const const_iterator& o) const { return i_ != o.i_; }
    bool operator==(const const_iterator& o) const { return i_ == o.i_; }

private:
    const Node* n_;
    std::size_t i_;
};

inline Node::const_iterator Node::begin() const { return const_iterator(this, 0); }
inline Node::const_iterator Node::end() const { return const_iterator(this, size()); }

template <>
inline std::string Node::as<std::string>() const
{
    if (!IsScalar()) throw TypedBadConversion(IsDefined() ? "<not a scalar>" : "<undefined>");
    return d_->scalar;
}

namespace detail {
template <class T>
inline T number(const Node& n, T (*conv)(const char*, char**))
{
    const std::string s = n.as<std::string>();
    if (s.empty()) throw TypedBadConversion(s);
    char* end = nullptr;
    errno = 0;
    const T v = conv(s.c_str(), &end);
    if (*end != '\0' || errno == ERANGE) throw TypedBadConversion(s);
    return v;
}
inline double to_double(const char* s, char** e) { return std::strtod(s, e); }
inline float to_float(const char* s, char** e) { return std::strtof(s, e); }
inline long long to_ll(const char* s, char** e) { return std::strtoll(s, e, 10); }
inline unsigned long long to_ull(const char* s, char** e) { return std::strtoull(s, e, 10); }
}  // namespace detail

template <>
inline double Node::as<double>() const { return detail::number<double>(*this, detail::to_double); }
template <>
inline float Node::as<float>() const { return detail::number<float>(*this, detail::to_float); }
template <>
inline int Node::as<int>() const { return (int)detail::number<long long>(*this, detail::to_ll); }
template <>
inline long Node::as<long>() const { return (long)detail::number<long long>(*this, detail::to_ll); }
template <>
inline long long Node::as<long long>() const { return detail::number<long long>(*this, detail::to_ll); }
template <>
inline unsigned long Node::as<unsigned long>() const
{
    return (unsigned long)detail::number<unsigned long long>(*this, detail::to_ull);
}
template <>
inline unsigned long long Node::as<unsigned long long>() const
{
    return detail::number<unsigned long long>(*this, detail::to_ull);
}
template <>
inline bool Node::as<bool>() const
{
    const std::string s = as<std::string>();
    if (s == "true" || s == "True" || s == "yes") return true;
    if (s == "false" || s == "False" || s == "no") return false;
    throw TypedBadConversion(s);
}

namespace detail {

struct Line {
    int number, indent;
    std::string text;    // without indentation and comment
};

inline std::string trim(const std::string& s)
{
    const auto b = s.find_first_not_of(" \t\r");
    if (b == std::string::npos) return "";
    const auto e = s.find_last_not_of(" \t\r");
    return s.substr(b, e - b + 1);
}

inline std::string strip_comment(const std::string& s)
{
    char q = 0;
    for (std::size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (q) {
            if (c == q) q = 0;
        } else if (c == '"' || c == '\'') {
            q = c;
        } else if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) {
            return s.substr(0, i);
        }
    }
    return s;
}

inline Node scalar(const std::string& raw)
{
    const std::string t = trim(raw);
    if (t.empty() || t == "~" || t == "null") return Node(NodeType::Null);
    if (t.size() >= 2 && (t.front() == '"' || t.front() == '\'') && t.back() == t.front())
        return Node(t.substr(1, t.size() - 2));
    return Node(t);
}

// flow collections and scalars: [..], {..}, plain
class Flow {
public:
    Flow(const std::string& s, int line) : s_(s), line_(line) {}
    Node parse()
    {
        Node n = value(",]}");
        skip();
        if (p_ != s_.size()) throw ParserException(line_, "trailing characters in '" + s_ + "'");
        return n;
    }

private:
    void skip()
    {
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t')) ++p_;
    }
    Node value(const char* stops)
    {
        skip();
        if (p_ < s_.size() && s_[p_] == '[') {
            ++p_;
            Node n(NodeType::Sequence);
            skip();
            if (p_ < s_.size() && s_[p_] == ']') { ++p_; return n; }
            for (;;) {
                n.push_back(value(",]"));
                skip();
                if (p_ >= s_.size()) throw ParserException(line_, "unterminated '['");
                if (s_[p_] == ',') { ++p_; continue; }
                if (s_[p_] == ']') { ++p_; return n; }
                throw ParserException(line_, "expected ',' or ']'");
            }
        }
        if (p_ < s_.size() && s_[p_] == '{') {
            ++p_;
            Node n(NodeType::Map);
            skip();
            if (p_ < s_.size() && s_[p_] == '}') { ++p_; return n; }
            for (;;) {
                const std::size_t k0 = p_;
                while (p_ < s_.size() && s_[p_] != ':' && s_[p_] != '}' && s_[p_] != ',') ++p_;
                if (p_ >= s_.size() || s_[p_] != ':') throw ParserException(line_, "expected ':' in a flow map");
                const Node key = scalar(s_.substr(k0, p_ - k0));
                ++p_;
                n.add(key, value(",}"));
                skip();
                if (p_ >= s_.size()) throw ParserException(line_, "unterminated '{'");
                if (s_[p_] == ',') { ++p_; skip(); continue; }
                if (s_[p_] == '}') { ++p_; return n; }
                throw ParserException(line_, "expected ',' or '}'");
            }
        }
        const std::size_t b = p_;
        char q = 0;
        while (p_ < s_.size()) {
            const char c = s_[p_];
            if (q) {
                if (c == q) q = 0;
            } else if (c == '"' || c == '\'') {
                q = c;
            } else if (std::string(stops).find(c) != std::string::npos) {
                break;
            }
            ++p_;
        }
        return scalar(s_.substr(b, p_ - b));
    }

    const std::string& s_;
    std::size_t p_ = 0;
    int line_;
};

inline Node inline_value(const std::string& v, int line)
{
    const std::string t = trim(v);
    if (!t.empty() && (t[0] == '[' || t[0] == '{')) return Flow(t, line).parse();
    return scalar(t);
}

// position of the ':' that ends a block-map key on this line, or npos
inline std::size_t key_colon(const std::string& t)
{
    char q = 0;
    for (std::size_t i = 0; i < t.size(); ++i) {
        const char c = t[i];
        if (q) {
            if (c == q) q = 0;
        } else if (c == '"' || c == '\'') {
            q = c;
        } else if (c == '[' || c == '{') {
            return std::string::npos;
        } else if (c == ':' && (i + 1 == t.size() || t[i + 1] == ' ' || t[i + 1] == '\t')) {
            return i;
        }
    }
    return std::string::npos;
}

class Block {
public:
    explicit Block(std::vector<Line> lines) : L_(std::move(lines)) {}
    Node document()
    {
        if (L_.empty()) return Node(NodeType::Null);
        Node n = node(L_[0].indent);
        if (i_ != L_.size()) throw ParserException(L_[i_].number, "unexpected indentation");
        return n;
    }

private:
    bool is_item(const Line& l) const { return l.text == "-" || l.text.compare(0, 2, "- ") == 0; }

    Node node(int indent)
    {
        if (is_item(L_[i_])) return sequence(indent);
        return map(indent);
    }

    // value of "key:" with nothing after it: a nested block (deeper, or a
    // sequence at the key's own indentation), else null
    Node nested(int key_indent)
    {
        if (i_ < L_.size() && (L_[i_].indent > key_indent || (L_[i_].indent == key_indent && is_item(L_[i_]))))
            return node(L_[i_].indent);
        return Node(NodeType::Null);
    }

    Node map(int indent)
    {
        Node m(NodeType::Map);
        while (i_ < L_.size() && L_[i_].indent == indent && !is_item(L_[i_])) {
            const Line& l = L_[i_];
            const std::size_t c = key_colon(l.text);
            if (c == std::string::npos) throw ParserException(l.number, "expected 'key: value'");
            const Node key = scalar(l.text.substr(0, c));
            const std::string rest = trim(l.text.substr(c + 1));
            ++i_;
            m.add(key, rest.empty() ? nested(indent) : inline_value(rest, l.number));
        }
        return m;
    }

    Node sequence(int indent)
    {
        Node s(NodeType::Sequence);
        while (i_ < L_.size() && L_[i_].indent == indent && is_item(L_[i_])) {
            Line& l = L_[i_];
            const std::string rest = l.text == "-" ? "" : l.text.substr(2);
            const std::string t = trim(rest);
            if (t.empty()) {
                ++i_;
                s.push_back(nested(indent));
            } else if (key_colon(t) != std::string::npos || t.compare(0, 2, "- ") == 0 || t == "-") {
                // an item that is itself a block: re-read this line as its first line,
                // indented where its text starts
                l.indent = indent + 2 + (int)rest.find_first_not_of(' ');
                l.text = t;
                s.push_back(node(l.indent));
            } else {
                ++i_;
                s.push_back(inline_value(t, l.number));
            }
        }
        return s;
    }

    std::vector<Line> L_;
    std::size_t i_ = 0;
};

inline std::vector<Line> lines_of(std::istream& in)
{
    std::vector<Line> out;
    std::string raw;
    int number = 0;
    while (std::getline(in, raw)) {
        ++number;
        const std::string s = strip_comment(raw);
        const std::string t = trim(s);
        if (t.empty() || t == "---" || t == "...") continue;
        const int indent = (int)s.find_first_not_of(' ');
        if (s[indent] == '\t') throw ParserException(number, "tab indentation");
        out.push_back({ number, indent, t });
    }
    return out;
}

}  // namespace detail

inline Node Load(const std::string& text)
{
    std::istringstream in(text);
    return detail::Block(detail::lines_of(in)).document();
}

inline Node LoadFile(const std::string& path)
{
    std::ifstream in(path);
    if (!in) throw BadFile(path);
    return detail::Block(detail::lines_of(in)).document();
}

}  // namespace YAML
