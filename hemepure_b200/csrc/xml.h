// xml.h -- minimal XML DOM for HemeLB case files (the reference wraps tinyxml in
// src/io/xml/XmlAbstractionLayer.{h,cc}; only elements and attributes matter).
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace hb {

struct XmlElement {
  std::string name;
  std::map<std::string, std::string> attrs;
  std::vector<std::unique_ptr<XmlElement>> children;
  int line = 0;

  // First child named `n`, or nullptr (Element::GetChildOrNull).
  const XmlElement* child(const std::string& n) const;
  // First child named `n`; throws hb::Error(HB_ERR_FORMAT) when absent (GetChildOrThrow).
  const XmlElement& require(const std::string& n) const;
  std::vector<const XmlElement*> all(const std::string& n) const;
  // Attribute value; throws when absent (GetAttributeOrThrow).
  const std::string& attr(const std::string& a) const;
  bool has(const std::string& a) const { return attrs.count(a) != 0; }
};

// Parse a document; throws hb::Error on malformed input.
std::unique_ptr<XmlElement> xml_parse(const std::string& text);
std::unique_ptr<XmlElement> xml_parse_file(const std::string& path);

}  // namespace hb
