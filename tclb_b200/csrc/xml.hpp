// Minimal XML reader for TCLB case files (<CLBConfig>): elements, attributes,
// comments, processing instructions and the five predefined entities. Text
// content is ignored (TCLB cases carry everything in attributes).
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace tclb {

struct XmlNode {
  std::string name;
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<std::unique_ptr<XmlNode>> children;
  XmlNode* parent = nullptr;

  const std::string* attr(const std::string& k) const {
    for (const auto& a : attrs)
      if (a.first == k) return &a.second;
    return nullptr;
  }
  std::string attr_or(const std::string& k, const std::string& d) const {
    const std::string* v = attr(k);
    return v ? *v : d;
  }
  const XmlNode* child(const std::string& n) const {
    for (const auto& c : children)
      if (c->name == n) return c.get();
    return nullptr;
  }
  const XmlNode* child_by_attr(const std::string& n, const std::string& k, const std::string& v) const {
    for (const auto& c : children)
      if (c->name == n) {
        const std::string* a = c->attr(k);
        if (a && *a == v) return c.get();
      }
    return nullptr;
  }
};

class XmlParser {
 public:
  explicit XmlParser(const std::string& text) : s_(text) {}

  std::unique_ptr<XmlNode> parse() {
    auto doc = std::make_unique<XmlNode>();
    doc->name = "#document";
    parse_content(doc.get(), true);
    return doc;
  }

 private:
  const std::string& s_;
  size_t p_ = 0;

  [[noreturn]] void error(const std::string& msg) const {
    size_t line = 1;
    for (size_t i = 0; i < p_ && i < s_.size(); i++) line += s_[i] == '\n';
    throw std::runtime_error("XML line " + std::to_string(line) + ": " + msg);
  }
  bool starts(const char* t) const { return s_.compare(p_, std::char_traits<char>::length(t), t) == 0; }
  void skip_ws() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) p_++;
  }
  void skip_past(const char* t) {
    size_t q = s_.find(t, p_);
    if (q == std::string::npos) error(std::string("unterminated construct, expected ") + t);
    p_ = q + std::char_traits<char>::length(t);
  }
  static bool name_char(char c) {
    return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' || c == '-' ||
           c == '.' || c == ':';
  }
  std::string name() {
    size_t b = p_;
    while (p_ < s_.size() && name_char(s_[p_])) p_++;
    if (p_ == b) error("expected a name");
    return s_.substr(b, p_ - b);
  }
  std::string unescape(const std::string& v) {
    std::string o;
    for (size_t i = 0; i < v.size(); i++) {
      if (v[i] != '&') {
        o += v[i];
        continue;
      }
      size_t e = v.find(';', i);
      if (e == std::string::npos) error("bad entity");
      const std::string ent = v.substr(i + 1, e - i - 1);
      if (ent == "lt") o += '<';
      else if (ent == "gt") o += '>';
      else if (ent == "amp") o += '&';
      else if (ent == "quot") o += '"';
      else if (ent == "apos") o += '\'';
      else if (!ent.empty() && ent[0] == '#') o += (char)std::stoi(ent[1] == 'x' ? "0" + ent.substr(1) : ent.substr(1), nullptr, ent[1] == 'x' ? 16 : 10);
      else error("unknown entity &" + ent + ";");
      i = e;
    }
    return o;
  }
  void parse_content(XmlNode* parent, bool top) {
    while (p_ < s_.size()) {
      if (starts("<!--")) {
        skip_past("-->");
      } else if (starts("<?")) {
        skip_past("?>");
      } else if (starts("<!")) {
        skip_past(">");
      } else if (starts("</")) {
        if (top) error("unexpected closing tag");
        p_ += 2;
        const std::string n = name();
        if (n != parent->name) error("closing tag </" + n + "> does not match <" + parent->name + ">");
        skip_ws();
        if (p_ >= s_.size() || s_[p_] != '>') error("expected >");
        p_++;
        return;
      } else if (s_[p_] == '<') {
        p_++;
        auto node = std::make_unique<XmlNode>();
        node->name = name();
        node->parent = parent;
        for (;;) {
          skip_ws();
          if (p_ >= s_.size()) error("unterminated tag");
          if (s_[p_] == '/') {
            p_++;
            if (p_ >= s_.size() || s_[p_] != '>') error("expected />");
            p_++;
            break;
          }
          if (s_[p_] == '>') {
            p_++;
            parse_content(node.get(), false);
            break;
          }
          const std::string k = name();
          skip_ws();
          if (p_ >= s_.size() || s_[p_] != '=') error("expected = after attribute " + k);
          p_++;
          skip_ws();
          if (p_ >= s_.size() || (s_[p_] != '"' && s_[p_] != '\'')) error("expected quoted value");
          const char q = s_[p_++];
          size_t e = s_.find(q, p_);
          if (e == std::string::npos) error("unterminated attribute value");
          node->attrs.emplace_back(k, unescape(s_.substr(p_, e - p_)));
          p_ = e + 1;
        }
        parent->children.push_back(std::move(node));
      } else {
        p_++;  // text content: ignored
      }
    }
    if (!top) error("unterminated element <" + parent->name + ">");
  }
};

}  // namespace tclb
