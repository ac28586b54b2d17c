// Report templating is not on the collide-and-stream path; this stand-in for
// ctemplate keeps the reference's reporting code compiling and records nothing
// (CPU oracle build only).
#ifndef HB_REF_SHIM_CTEMPLATE_TEMPLATE_H
#define HB_REF_SHIM_CTEMPLATE_TEMPLATE_H
#include <list>
#include <string>
namespace ctemplate {
enum Strip { DO_NOT_STRIP, STRIP_BLANK_LINES, STRIP_WHITESPACE };
class TemplateDictionary {
 public:
  explicit TemplateDictionary(const std::string& = std::string()) {}
  void SetValue(const std::string&, const std::string&) {}
  void SetIntValue(const std::string&, long) {}
  void SetFormattedValue(const std::string&, const char*, ...) {}
  TemplateDictionary* AddSectionDictionary(const std::string&) {
    children_.emplace_back();
    return &children_.back();
  }
  void ShowSection(const std::string&) {}

 private:
  std::list<TemplateDictionary> children_;
};
inline bool ExpandTemplate(const std::string&, Strip, const TemplateDictionary*, std::string* out) {
  if (out) out->clear();
  return true;
}
}  // namespace ctemplate
#endif
