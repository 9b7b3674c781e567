// Minimal stand-in for yaml-cpp (not installed here), for the oracle/_ref build only. pirate's
// reference CPU path never parses or emits YAML when its configs are built in code, so Node is an
// always-undefined node whose conversions throw, and Emitter discards what it is given.
#ifndef _YAML_CPP_SHIM_YAML_H
#define _YAML_CPP_SHIM_YAML_H

#include <cstddef>
#include <stdexcept>
#include <string>

namespace YAML {

struct NodeType { enum value { Undefined, Null, Scalar, Sequence, Map }; };

enum EMITTER_MANIP { BeginMap, EndMap, BeginSeq, EndSeq, Key, Value, Flow, Block, Newline, Auto };

struct _Comment { std::string s; };
inline _Comment Comment(const std::string &s) { return _Comment{s}; }

class Node
{
public:
    Node() {}
    NodeType::value Type() const { return NodeType::Undefined; }
    bool IsDefined() const { return false; }
    bool IsNull() const { return false; }
    bool IsScalar() const { return false; }
    bool IsSequence() const { return false; }
    bool IsMap() const { return false; }
    explicit operator bool() const { return false; }
    bool operator!() const { return true; }
    std::size_t size() const { return 0; }
    template<typename K> Node operator[](const K &) const { return Node(); }
    template<typename T> T as() const { throw std::runtime_error("yaml-cpp shim: YAML parsing is not available in this shim"); }
    const std::string &Scalar() const { static std::string s; return s; }
    struct iterator {
        bool operator!=(const iterator &) const { return false; }
        iterator &operator++() { return *this; }
        std::pair<Node, Node> operator*() const { return {Node(), Node()}; }
        const std::pair<Node, Node> *operator->() const { static std::pair<Node, Node> p; return &p; }
    };
    iterator begin() const { return iterator(); }
    iterator end() const { return iterator(); }
};

inline Node Load(const std::string &) { throw std::runtime_error("yaml-cpp shim: YAML parsing is not available in this shim"); }
inline Node LoadFile(const std::string &) { throw std::runtime_error("yaml-cpp shim: YAML parsing is not available in this shim"); }

class Emitter
{
public:
    template<typename T> Emitter &operator<<(const T &) { return *this; }
    const char *c_str() const { return ""; }
    std::size_t size() const { return 0; }
    bool good() const { return true; }
    std::string GetLastError() const { return ""; }
    Emitter &SetIndent(int) { return *this; }
    Emitter &SetDoublePrecision(int) { return *this; }
    Emitter &SetFloatPrecision(int) { return *this; }
};

}  // namespace YAML

#endif
