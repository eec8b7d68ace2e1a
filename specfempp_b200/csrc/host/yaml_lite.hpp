// A small YAML reader for the reference's parameter, source and station files:
// block mappings and sequences by indentation, flow-free scalars, quoted
// strings, `#` comments and `|` / `>` block scalars.  It covers the subset the
// reference's files use (parameter_files/, tests/unit-tests/*/specfem_config.yaml,
// sources.yaml); anchors, tags and flow collections are rejected.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace sfb {

struct YNode {
  enum Kind { NONE, SCALAR, MAP, SEQ } kind = NONE;
  std::string scalar;
  std::vector<std::pair<std::string, std::shared_ptr<YNode>>> map;
  std::vector<std::shared_ptr<YNode>> seq;

  bool is_map() const { return kind == MAP; }
  bool is_seq() const { return kind == SEQ; }
  bool is_scalar() const { return kind == SCALAR; }
  // Child lookup; returns nullptr when absent (or when this is not a map).
  const YNode *get(const std::string &key) const;
  const YNode *path(const std::vector<std::string> &keys) const;
  std::string str() const;
  double num() const;
  int integer() const;
  bool boolean() const;
};

std::shared_ptr<YNode> yaml_parse(const std::string &text);
std::shared_ptr<YNode> yaml_load_file(const std::string &path);

}  // namespace sfb
