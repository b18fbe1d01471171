// Minimal XML document reader for ARTSS input files.
//
// Supports what ARTSS inputs use: the XML declaration, comments, elements
// with quoted attributes, self-closing elements, text content and the five
// predefined entities.  Text of an element is its first text run, like
// tinyxml2's XMLElement::GetText() which the reference settings parser reads
// (ARTSS src/utility/settings/Settings.cpp:40-53).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace artss {

struct XmlElement {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attributes;  // in document order
    std::string text;       // first text run
    bool has_text = false;
    std::vector<std::unique_ptr<XmlElement>> children;

    const XmlElement *first_child(const std::string &child_name) const;
    const std::string *attribute(const std::string &key) const;
};

class XmlError : public std::runtime_error {
 public:
    explicit XmlError(const std::string &m) : std::runtime_error(m) {}
};

// Parses a whole document and returns its root element.
std::unique_ptr<XmlElement> parse_xml(const std::string &content);

}  // namespace artss
