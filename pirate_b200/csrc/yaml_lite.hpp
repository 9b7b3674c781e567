// yaml_lite.hpp -- a small YAML-subset reader for dedispersion config files.
//
// Supports what pirate's configs use (configs/dedispersion/*.yml): block mappings, block sequences,
// flow sequences "[a, b]", flow mappings "{k: v, ...}", plain/quoted scalars and '#' comments.
// Anchors, tags, multi-document streams and block scalars are not supported (they raise errors).

#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace pb2 {
namespace yaml {

struct Node
{
    enum Kind { Null, Scalar, Seq, Map } kind = Null;
    std::string scalar;
    std::vector<std::shared_ptr<Node>> seq;
    std::vector<std::pair<std::string, std::shared_ptr<Node>>> map;   // insertion order kept

    const Node *get(const std::string &key) const
    {
        for (auto &kv : map)
            if (kv.first == key) return kv.second.get();
        return nullptr;
    }
};

using NodeP = std::shared_ptr<Node>;

class Parser
{
public:
    explicit Parser(const std::string &text, const std::string &name) : name_(name) { split_lines(text); }

    NodeP parse()
    {
        size_t i = 0;
        skip_blank(i);
        if (i >= lines_.size()) return std::make_shared<Node>();
        NodeP n = parse_block(i, lines_[i].indent);
        skip_blank(i);
        if (i < lines_.size()) fail(i, "unexpected content");
        return n;
    }

private:
    struct Line { int indent; std::string text; int lineno; };
    std::vector<Line> lines_;
    std::string name_;

    [[noreturn]] void fail(size_t i, const std::string &why) const
    {
        int ln = (i < lines_.size()) ? lines_[i].lineno : -1;
        throw std::runtime_error(name_ + ":" + std::to_string(ln) + ": yaml parse error: " + why);
    }

    static std::string strip_comment(const std::string &s)
    {
        bool sq = false, dq = false;
        for (size_t k = 0; k < s.size(); k++) {
            char c = s[k];
            if (c == '\'' && !dq) sq = !sq;
            else if (c == '"' && !sq) dq = !dq;
            else if (c == '#' && !sq && !dq && (k == 0 || s[k-1] == ' ' || s[k-1] == '\t')) return s.substr(0, k);
        }
        return s;
    }

    static std::string trim(const std::string &s)
    {
        size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
        return (a == std::string::npos) ? std::string() : s.substr(a, b - a + 1);
    }

    void split_lines(const std::string &text)
    {
        size_t pos = 0;
        int ln = 0;
        while (pos <= text.size()) {
            size_t e = text.find('\n', pos);
            if (e == std::string::npos) e = text.size();
            std::string raw = text.substr(pos, e - pos);
            ln++;
            pos = e + 1;
            if (raw.find('\t') != std::string::npos && trim(strip_comment(raw)).size() && raw.find_first_not_of(" \t") > raw.find('\t'))
                throw std::runtime_error(name_ + ":" + std::to_string(ln) + ": tabs are not allowed for indentation");
            std::string t = strip_comment(raw);
            std::string tt = trim(t);
            if (tt.empty() || tt == "---") continue;
            int ind = (int) t.find_first_not_of(' ');
            lines_.push_back({ind, tt, ln});
            if (e == text.size()) break;
        }
    }

    void skip_blank(size_t &) const { }

    // Splits "key: rest" at the first ':' outside quotes/brackets followed by space or end.
    static bool split_key(const std::string &s, std::string &key, std::string &rest)
    {
        int depth = 0;
        bool sq = false, dq = false;
        for (size_t k = 0; k < s.size(); k++) {
            char c = s[k];
            if (c == '\'' && !dq) sq = !sq;
            else if (c == '"' && !sq) dq = !dq;
            else if (sq || dq) continue;
            else if (c == '[' || c == '{') depth++;
            else if (c == ']' || c == '}') depth--;
            else if (c == ':' && depth == 0 && (k + 1 == s.size() || s[k+1] == ' ')) {
                key = unquote(trim(s.substr(0, k)));
                rest = trim(s.substr(k + 1));
                return true;
            }
        }
        return false;
    }

    static std::string unquote(const std::string &s)
    {
        if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
            return s.substr(1, s.size() - 2);
        return s;
    }

    NodeP parse_block(size_t &i, int indent)
    {
        if (i >= lines_.size()) return std::make_shared<Node>();
        const std::string &t = lines_[i].text;
        if (t[0] == '-' && (t.size() == 1 || t[1] == ' '))
            return parse_seq(i, indent);
        return parse_map(i, indent);
    }

    NodeP parse_seq(size_t &i, int indent)
    {
        auto n = std::make_shared<Node>();
        n->kind = Node::Seq;
        while (i < lines_.size() && lines_[i].indent == indent) {
            const std::string &t = lines_[i].text;
            if (!(t[0] == '-' && (t.size() == 1 || t[1] == ' '))) break;
            std::string rest = trim(t.substr(1));
            if (rest.empty()) {
                i++;
                if (i < lines_.size() && lines_[i].indent > indent) n->seq.push_back(parse_block(i, lines_[i].indent));
                else n->seq.push_back(std::make_shared<Node>());
                continue;
            }
            std::string key, val;
            if ((rest[0] != '[' && rest[0] != '{' && rest[0] != '"' && rest[0] != '\'') && split_key(rest, key, val)) {
                // "- key: val" starts a block mapping whose continuation lines are indented further.
                int sub_indent = indent + (int) (t.size() - rest.size());
                lines_[i].indent = sub_indent;
                lines_[i].text = rest;
                n->seq.push_back(parse_map(i, sub_indent));
                continue;
            }
            size_t p = 0;
            n->seq.push_back(parse_flow(rest, p, i));
            if (trim(rest.substr(p)).size()) fail(i, "trailing characters after flow value");
            i++;
        }
        return n;
    }

    NodeP parse_map(size_t &i, int indent)
    {
        auto n = std::make_shared<Node>();
        n->kind = Node::Map;
        while (i < lines_.size() && lines_[i].indent == indent) {
            std::string key, rest;
            if (!split_key(lines_[i].text, key, rest)) fail(i, "expected 'key: value'");
            if (n->get(key)) fail(i, "duplicate key '" + key + "'");
            size_t here = i;
            i++;
            NodeP v;
            if (rest.empty()) {
                if (i < lines_.size() && lines_[i].indent > indent) v = parse_block(i, lines_[i].indent);
                else if (i < lines_.size() && lines_[i].indent == indent && lines_[i].text[0] == '-') v = parse_seq(i, indent);
                else v = std::make_shared<Node>();
            }
            else {
                if (rest[0] == '|' || rest[0] == '>' || rest[0] == '&' || rest[0] == '*' || rest[0] == '!')
                    fail(here, "unsupported yaml feature");
                size_t p = 0;
                v = parse_flow(rest, p, here);
                if (trim(rest.substr(p)).size()) fail(here, "trailing characters after value");
            }
            n->map.push_back({key, v});
        }
        if (i < lines_.size() && lines_[i].indent > indent) fail(i, "bad indentation");
        return n;
    }

    NodeP parse_flow(const std::string &s, size_t &p, size_t li)
    {
        while (p < s.size() && s[p] == ' ') p++;
        if (p >= s.size()) fail(li, "missing value");
        if (s[p] == '[' || s[p] == '{') {
            bool is_seq = (s[p] == '[');
            char close = is_seq ? ']' : '}';
            auto n = std::make_shared<Node>();
            n->kind = is_seq ? Node::Seq : Node::Map;
            p++;
            for (;;) {
                while (p < s.size() && s[p] == ' ') p++;
                if (p >= s.size()) fail(li, "unterminated flow collection");
                if (s[p] == close) { p++; break; }
                if (is_seq) n->seq.push_back(parse_flow(s, p, li));
                else {
                    size_t k0 = p;
                    while (p < s.size() && s[p] != ':') p++;
                    if (p >= s.size()) fail(li, "expected ':' in flow mapping");
                    std::string key = unquote(trim(s.substr(k0, p - k0)));
                    p++;
                    n->map.push_back({key, parse_flow(s, p, li)});
                }
                while (p < s.size() && s[p] == ' ') p++;
                if (p < s.size() && s[p] == ',') { p++; continue; }
                if (p < s.size() && s[p] == close) { p++; break; }
                fail(li, "expected ',' or closing bracket");
            }
            return n;
        }
        auto n = std::make_shared<Node>();
        n->kind = Node::Scalar;
        if (s[p] == '"' || s[p] == '\'') {
            char q = s[p];
            size_t e = s.find(q, p + 1);
            if (e == std::string::npos) fail(li, "unterminated quoted scalar");
            n->scalar = s.substr(p + 1, e - p - 1);
            p = e + 1;
            return n;
        }
        size_t e = p;
        while (e < s.size() && s[e] != ',' && s[e] != ']' && s[e] != '}') e++;
        n->scalar = trim(s.substr(p, e - p));
        p = e;
        if (n->scalar == "~" || n->scalar == "null") n->kind = Node::Null;
        return n;
    }
};

inline NodeP parse(const std::string &text, const std::string &name = "yaml")
{
    return Parser(text, name).parse();
}

}  // namespace yaml
}  // namespace pb2
