#include "xml.h"

#include <cctype>
#include <cstring>

namespace artss {

const XmlElement *XmlElement::first_child(const std::string &child_name) const {
    for (const auto &c : children)
        if (c->name == child_name) return c.get();
    return nullptr;
}

const std::string *XmlElement::attribute(const std::string &key) const {
    for (const auto &kv : attributes)
        if (kv.first == key) return &kv.second;
    return nullptr;
}

namespace {

class Parser {
 public:
    explicit Parser(const std::string &s) : s_(s) {}

    std::unique_ptr<XmlElement> document() {
        skip_misc();
        if (!peek("<")) fail("no root element");
        auto root = element();
        skip_misc();
        return root;
    }

 private:
    const std::string &s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string &what) const {
        size_t line = 1;
        for (size_t q = 0; q < p_ && q < s_.size(); q++) line += s_[q] == '\n';
        throw XmlError("XML parse error at line " + std::to_string(line) + ": " + what);
    }
    bool eof() const { return p_ >= s_.size(); }
    bool peek(const char *t) const { return s_.compare(p_, std::strlen(t), t) == 0; }
    void expect(const char *t) {
        if (!peek(t)) fail(std::string("expected '") + t + "'");
        p_ += std::strlen(t);
    }
    void skip_ws() {
        while (!eof() && std::isspace(static_cast<unsigned char>(s_[p_]))) p_++;
    }
    void skip_until(const char *t) {
        size_t q = s_.find(t, p_);
        if (q == std::string::npos) fail(std::string("unterminated construct, missing '") + t + "'");
        p_ = q + std::strlen(t);
    }
    // whitespace, comments, declarations, processing instructions, DOCTYPE
    void skip_misc() {
        for (;;) {
            skip_ws();
            if (peek("<!--")) skip_until("-->");
            else if (peek("<?")) skip_until("?>");
            else if (peek("<!")) skip_until(">");
            else break;
        }
    }
    static bool name_char(char c) {
        return std::isalnum(static_cast<unsigned char>(c)) || c == '_' || c == '-' || c == '.' || c == ':';
    }
    std::string name() {
        size_t b = p_;
        while (!eof() && name_char(s_[p_])) p_++;
        if (b == p_) fail("expected a name");
        return s_.substr(b, p_ - b);
    }
    std::string decode(const std::string &raw) const {
        std::string out;
        out.reserve(raw.size());
        for (size_t q = 0; q < raw.size(); q++) {
            if (raw[q] != '&') { out += raw[q]; continue; }
            size_t e = raw.find(';', q);
            if (e == std::string::npos) { out += raw[q]; continue; }
            std::string ent = raw.substr(q + 1, e - q - 1);
            if (ent == "lt") out += '<';
            else if (ent == "gt") out += '>';
            else if (ent == "amp") out += '&';
            else if (ent == "quot") out += '"';
            else if (ent == "apos") out += '\'';
            else if (!ent.empty() && ent[0] == '#') {
                long v = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X') ? std::strtol(ent.c_str() + 2, nullptr, 16)
                                                                          : std::strtol(ent.c_str() + 1, nullptr, 10);
                if (v > 0 && v < 128) out += static_cast<char>(v);
            } else {
                out += raw.substr(q, e - q + 1);
            }
            q = e;
        }
        return out;
    }
    std::unique_ptr<XmlElement> element() {
        expect("<");
        auto el = std::make_unique<XmlElement>();
        el->name = name();
        for (;;) {
            skip_ws();
            if (peek("/>")) { p_ += 2; return el; }
            if (peek(">")) { p_ += 1; break; }
            std::string key = name();
            skip_ws();
            expect("=");
            skip_ws();
            if (eof() || (s_[p_] != '"' && s_[p_] != '\'')) fail("attribute value must be quoted");
            const char q = s_[p_++];
            size_t e = s_.find(q, p_);
            if (e == std::string::npos) fail("unterminated attribute value");
            el->attributes.emplace_back(key, decode(s_.substr(p_, e - p_)));
            p_ = e + 1;
        }
        // content
        for (;;) {
            if (eof()) fail("unterminated element <" + el->name + ">");
            if (peek("</")) {
                p_ += 2;
                std::string n = name();
                if (n != el->name) fail("mismatched closing tag </" + n + "> for <" + el->name + ">");
                skip_ws();
                expect(">");
                return el;
            }
            if (peek("<!--")) { skip_until("-->"); continue; }
            if (peek("<![CDATA[")) {
                p_ += 9;
                size_t e = s_.find("]]>", p_);
                if (e == std::string::npos) fail("unterminated CDATA");
                if (!el->has_text) { el->text = s_.substr(p_, e - p_); el->has_text = true; }
                p_ = e + 3;
                continue;
            }
            if (peek("<?")) { skip_until("?>"); continue; }
            if (peek("<")) { el->children.push_back(element()); continue; }
            size_t e = s_.find('<', p_);
            if (e == std::string::npos) fail("unterminated element <" + el->name + ">");
            std::string raw = s_.substr(p_, e - p_);
            p_ = e;
            bool blank = true;
            for (char c : raw) blank = blank && std::isspace(static_cast<unsigned char>(c));
            // whitespace-only runs are not text (tinyxml2 drops them)
            if (!blank && !el->has_text) { el->text = decode(raw); el->has_text = true; }
        }
    }
};

}  // namespace

std::unique_ptr<XmlElement> parse_xml(const std::string &content) {
    Parser p(content);
    return p.document();
}

}  // namespace artss
