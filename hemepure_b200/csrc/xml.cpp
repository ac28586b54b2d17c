// xml.cpp -- minimal XML parser: elements, attributes, comments, prolog.
#include "xml.h"

#include <fstream>
#include <sstream>

#include "../../include/hemeb200.h"
#include "hb_common.h"

namespace hb {

const XmlElement* XmlElement::child(const std::string& n) const {
  for (auto& c : children)
    if (c->name == n) return c.get();
  return nullptr;
}

const XmlElement& XmlElement::require(const std::string& n) const {
  const XmlElement* c = child(n);
  if (!c) throw Error{HB_ERR_FORMAT, "missing element <" + n + "> under <" + name + ">"};
  return *c;
}

std::vector<const XmlElement*> XmlElement::all(const std::string& n) const {
  std::vector<const XmlElement*> out;
  for (auto& c : children)
    if (c->name == n) out.push_back(c.get());
  return out;
}

const std::string& XmlElement::attr(const std::string& a) const {
  auto it = attrs.find(a);
  if (it == attrs.end()) throw Error{HB_ERR_FORMAT, "missing attribute '" + a + "' on <" + name + ">"};
  return it->second;
}

namespace {

struct Parser {
  const std::string& s;
  size_t p = 0;
  int line = 1;

  [[noreturn]] void fail(const std::string& why) {
    throw Error{HB_ERR_FORMAT, "XML parse error at line " + std::to_string(line) + ": " + why};
  }
  bool eof() const { return p >= s.size(); }
  char peek() const { return p < s.size() ? s[p] : '\0'; }
  void adv(size_t k = 1) {
    for (size_t i = 0; i < k && p < s.size(); i++, p++)
      if (s[p] == '\n') line++;
  }
  bool starts(const char* t) const { return s.compare(p, std::char_traits<char>::length(t), t) == 0; }
  void skip_ws() {
    while (!eof() && (peek() == ' ' || peek() == '\t' || peek() == '\n' || peek() == '\r')) adv();
  }
  void skip_until(const char* t) {
    size_t k = s.find(t, p);
    if (k == std::string::npos) fail(std::string("unterminated construct, expected ") + t);
    adv(k - p + std::char_traits<char>::length(t));
  }
  // Skip text, comments, processing instructions and doctype between elements.
  void skip_misc() {
    for (;;) {
      while (!eof() && peek() != '<') adv();
      if (eof()) return;
      if (starts("<!--")) skip_until("-->");
      else if (starts("<?")) skip_until("?>");
      else if (starts("<!")) skip_until(">");
      else return;
    }
  }
  std::string name() {
    size_t b = p;
    while (!eof() && (isalnum((unsigned char)peek()) || peek() == '_' || peek() == '-' || peek() == ':' || peek() == '.')) adv();
    if (p == b) fail("expected a name");
    return s.substr(b, p - b);
  }
  static std::string unescape(const std::string& v) {
    std::string o;
    for (size_t i = 0; i < v.size(); i++) {
      if (v[i] == '&') {
        size_t e = v.find(';', i);
        std::string ent = e == std::string::npos ? "" : v.substr(i, e - i + 1);
        if (ent == "&lt;") o += '<';
        else if (ent == "&gt;") o += '>';
        else if (ent == "&amp;") o += '&';
        else if (ent == "&quot;") o += '"';
        else if (ent == "&apos;") o += '\'';
        else {
          o += v[i];
          continue;
        }
        i = e;
      } else {
        o += v[i];
      }
    }
    return o;
  }
  std::unique_ptr<XmlElement> element() {
    if (peek() != '<') fail("expected '<'");
    adv();
    auto el = std::make_unique<XmlElement>();
    el->line = line;
    el->name = name();
    for (;;) {
      skip_ws();
      if (starts("/>")) {
        adv(2);
        return el;
      }
      if (peek() == '>') {
        adv();
        break;
      }
      std::string an = name();
      skip_ws();
      if (peek() != '=') fail("expected '=' after attribute " + an);
      adv();
      skip_ws();
      char q = peek();
      if (q != '"' && q != '\'') fail("expected a quoted attribute value");
      adv();
      size_t b = p;
      while (!eof() && peek() != q) adv();
      if (eof()) fail("unterminated attribute value");
      el->attrs[an] = unescape(s.substr(b, p - b));
      adv();
    }
    for (;;) {
      skip_misc();
      if (eof()) fail("unterminated element <" + el->name + ">");
      if (starts("</")) {
        adv(2);
        std::string cn = name();
        if (cn != el->name) fail("mismatched closing tag </" + cn + "> for <" + el->name + ">");
        skip_ws();
        if (peek() != '>') fail("expected '>'");
        adv();
        return el;
      }
      el->children.push_back(element());
    }
  }
};

}  // namespace

std::unique_ptr<XmlElement> xml_parse(const std::string& text) {
  Parser ps{text};
  ps.skip_misc();
  if (ps.eof()) throw Error{HB_ERR_FORMAT, "XML document has no root element"};
  return ps.element();
}

std::unique_ptr<XmlElement> xml_parse_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error{HB_ERR_IO, "cannot open " + path};
  std::stringstream ss;
  ss << in.rdbuf();
  return xml_parse(ss.str());
}

}  // namespace hb
