#include "yaml_lite.hpp"

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace sfb {

namespace {

struct Line {
  int indent;
  std::string text;  // without indentation and comments, right-trimmed
  std::string raw;   // original line (for block scalars)
};

std::string rtrim(const std::string &s) {
  size_t e = s.find_last_not_of(" \t\r");
  return e == std::string::npos ? std::string() : s.substr(0, e + 1);
}
std::string trim(const std::string &s) {
  size_t b = s.find_first_not_of(" \t\r");
  if (b == std::string::npos) return std::string();
  return rtrim(s.substr(b));
}

std::string strip_comment(const std::string &s) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (c == '#' && !sq && !dq && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t'))
      return s.substr(0, i);
  }
  return s;
}

std::string unquote(const std::string &s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') ||
                        (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}

// Position of the mapping colon ("key: value" or "key:"), or npos.
size_t find_colon(const std::string &s) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (c == ':' && !sq && !dq && (i + 1 == s.size() || s[i + 1] == ' ' || s[i + 1] == '\t'))
      return i;
  }
  return std::string::npos;
}

struct Parser {
  std::vector<Line> lines;
  size_t i = 0;

  std::shared_ptr<YNode> scalar(const std::string &v) {
    auto n = std::make_shared<YNode>();
    n->kind = YNode::SCALAR;
    n->scalar = unquote(trim(v));
    return n;
  }

  // Block scalar introduced by '|' or '>' on the previous line.
  std::shared_ptr<YNode> block_scalar(int parent_indent, bool folded) {
    std::string out;
    int block_indent = -1;
    while (i < lines.size()) {
      const Line &l = lines[i];
      if (l.indent <= parent_indent && !l.text.empty()) break;
      if (block_indent < 0) block_indent = l.indent;
      std::string t = l.raw.size() > static_cast<size_t>(block_indent)
                          ? rtrim(l.raw.substr(block_indent))
                          : std::string();
      if (!out.empty()) out += folded ? " " : "\n";
      out += t;
      ++i;
    }
    auto n = std::make_shared<YNode>();
    n->kind = YNode::SCALAR;
    n->scalar = out;
    return n;
  }

  std::shared_ptr<YNode> value_after_key(int indent, const std::string &rest) {
    const std::string v = trim(rest);
    if (v.empty()) {
      if (i < lines.size() &&
          (lines[i].indent > indent ||
           (lines[i].indent == indent && lines[i].text.rfind("-", 0) == 0 &&
            (lines[i].text.size() == 1 || lines[i].text[1] == ' '))))
        return block(lines[i].indent);
      return std::make_shared<YNode>();
    }
    if (v == "|" || v == "|-" || v == "|+") return block_scalar(indent, false);
    if (v == ">" || v == ">-" || v == ">+") return block_scalar(indent, true);
    if (v.front() == '[' || v.front() == '{') {
      // Flow sequence of scalars only: [a, b, c]
      if (v.front() == '[' && v.back() == ']') {
        auto n = std::make_shared<YNode>();
        n->kind = YNode::SEQ;
        std::stringstream ss(v.substr(1, v.size() - 2));
        std::string item;
        while (std::getline(ss, item, ','))
          if (!trim(item).empty()) n->seq.push_back(scalar(item));
        return n;
      }
      throw std::runtime_error("YAML flow mappings are not supported: " + v);
    }
    return scalar(v);
  }

  std::shared_ptr<YNode> block(int indent) {
    auto node = std::make_shared<YNode>();
    if (i >= lines.size()) return node;
    const bool is_seq = lines[i].text.rfind("-", 0) == 0 &&
                        (lines[i].text.size() == 1 || lines[i].text[1] == ' ');
    if (is_seq) {
      node->kind = YNode::SEQ;
      while (i < lines.size() && lines[i].indent == indent &&
             lines[i].text.rfind("-", 0) == 0 &&
             (lines[i].text.size() == 1 || lines[i].text[1] == ' ')) {
        std::string rest = lines[i].text.substr(1);
        const size_t off = rest.find_first_not_of(' ');
        if (off == std::string::npos) {
          ++i;
          if (i < lines.size() && lines[i].indent > indent)
            node->seq.push_back(block(lines[i].indent));
          else
            node->seq.push_back(std::make_shared<YNode>());
          continue;
        }
        // "- key: v" opens a mapping whose keys sit at indent + 1 + off.
        lines[i].indent = indent + 1 + static_cast<int>(off);
        lines[i].text = rest.substr(off);
        if (find_colon(lines[i].text) != std::string::npos) {
          node->seq.push_back(block(lines[i].indent));
        } else {
          node->seq.push_back(scalar(lines[i].text));
          ++i;
        }
      }
      return node;
    }
    node->kind = YNode::MAP;
    while (i < lines.size() && lines[i].indent == indent) {
      const std::string &t = lines[i].text;
      const size_t c = find_colon(t);
      if (c == std::string::npos) {
        if (node->map.empty()) {  // a bare scalar document
          auto s = scalar(t);
          ++i;
          return s;
        }
        throw std::runtime_error("YAML: expected 'key: value' in line: " + t);
      }
      const std::string key = unquote(trim(t.substr(0, c)));
      const std::string rest = t.substr(c + 1);
      ++i;
      node->map.emplace_back(key, value_after_key(indent, rest));
    }
    if (i < lines.size() && lines[i].indent > indent)
      throw std::runtime_error("YAML: unexpected indentation at: " + lines[i].text);
    return node;
  }
};

}  // namespace

const YNode *YNode::get(const std::string &key) const {
  if (kind != MAP) return nullptr;
  for (auto &kv : map)
    if (kv.first == key) return kv.second.get();
  return nullptr;
}

const YNode *YNode::path(const std::vector<std::string> &keys) const {
  const YNode *n = this;
  for (auto &k : keys) {
    n = n->get(k);
    if (!n) return nullptr;
  }
  return n;
}

std::string YNode::str() const {
  if (kind != SCALAR) throw std::runtime_error("YAML: expected a scalar");
  return scalar;
}
double YNode::num() const {
  const std::string s = str();
  char *end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw std::runtime_error("YAML: not a number: " + s);
  return v;
}
int YNode::integer() const { return static_cast<int>(num()); }
bool YNode::boolean() const {
  const std::string s = str();
  return s == "true" || s == "True" || s == "TRUE" || s == "yes" || s == "1";
}

std::shared_ptr<YNode> yaml_parse(const std::string &text) {
  Parser p;
  std::stringstream ss(text);
  std::string raw;
  while (std::getline(ss, raw)) {
    if (raw.find('\t') != std::string::npos && raw.find_first_not_of(" \t") != std::string::npos &&
        raw[raw.find_first_not_of(" ")] == '\t')
      throw std::runtime_error("YAML: tabs are not allowed for indentation");
    const std::string body = rtrim(strip_comment(raw));
    const size_t b = body.find_first_not_of(' ');
    Line l;
    l.raw = raw;
    if (b == std::string::npos) {
      // Blank / comment line: kept only inside block scalars.
      l.indent = 0;
      l.text.clear();
    } else {
      l.indent = static_cast<int>(b);
      l.text = body.substr(b);
    }
    if (l.text == "---" || l.text == "...") continue;
    p.lines.push_back(l);
  }
  // Drop blank lines (block scalars re-read raw text between non-blank ones).
  std::vector<Line> kept;
  for (auto &l : p.lines)
    if (!l.text.empty()) kept.push_back(l);
  p.lines = kept;
  if (p.lines.empty()) return std::make_shared<YNode>();
  return p.block(p.lines[0].indent);
}

std::shared_ptr<YNode> yaml_load_file(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("Could not open YAML file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return yaml_parse(ss.str());
}

}  // namespace sfb
