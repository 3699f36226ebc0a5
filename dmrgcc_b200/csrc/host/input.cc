// Input-file reader (see input.h).
#include "host/input.h"

#include <cctype>
#include <cstdio>

namespace dmrg {
namespace {

void eat_white(std::istream& is) {  // spaces, tabs, newlines
    char c;
    while (is.get(c))
        if (!std::isspace((unsigned char)c)) {
            is.putback(c);
            break;
        }
}

void eat_blank(std::istream& is) {  // spaces and tabs only
    char c;
    while (is.get(c))
        if (!std::isblank((unsigned char)c)) {
            is.putback(c);
            break;
        }
}

void match_bracket(std::istream& is) {
    int nest = 1;
    char c;
    while (is >> c) {
        if (c == '{') ++nest;
        else if (c == '}') --nest;
        if (nest == 0) return;
    }
    throw InputError("unterminated bracket");
}

// A token is a run of letters, '_' and (after the first character) digits, or
// one other character on its own.
bool get_token(std::istream& is, std::string& s) {
    eat_white(is);
    s.clear();
    char ch;
    for (int i = 0; i < 512; ++i) {
        if (!is.get(ch)) return !s.empty();
        if (std::isalpha((unsigned char)ch) || ch == '_' || (i != 0 && std::isdigit((unsigned char)ch))) {
            s.push_back(ch);
        } else {
            if (i == 0) {
                s.push_back(ch);
                return true;
            }
            is.putback(ch);
            break;
        }
    }
    return true;
}

// Skips the rest of the current line (brace groups on it are skipped whole).
void skip_rest_of_line(std::istream& is) {
    char c;
    while (is.get(c)) {
        if (c == '{') match_bracket(is);
        if (c == '\n') {
            eat_white(is);
            return;
        }
    }
}

}  // namespace

InputGroup::InputGroup(const std::string& file_name, const std::string& group_name, bool verbose)
    : file_name_(file_name), file_(std::make_shared<std::ifstream>()), name_(group_name), verbose_(verbose) {}

InputGroup::InputGroup(InputGroup& parent, const std::string& name)
    : file_name_(parent.file_name_), file_(parent.file_), parent_(&parent), name_(name), verbose_(parent.verbose_) {}

void InputGroup::reopen() {
    if (file_->is_open()) {
        file_->clear();
        file_->close();
    }
    file_->open(file_name_);
    if (!*file_) throw InputError("can't open input file " + file_name_);
}

bool InputGroup::GotoGroup() {
    if (parent_) parent_->GotoGroup();
    else reopen();
    std::istream& is = *file_;
    eat_white(is);
    for (;;) {
        std::string s;
        if (!get_token(is, s)) return false;
        if (s == name_) {
            eat_white(is);
            char c;
            is.get(c);
            if (c != '{') throw InputError("bracket does not follow group name " + name_);
            eat_white(is);
            return true;
        }
        if (s[0] == '{') match_bracket(is);
        skip_rest_of_line(is);
    }
}

bool InputGroup::GotoToken(const std::string& key) {
    if (!GotoGroup()) return false;
    std::istream& is = *file_;
    for (;;) {
        std::string t;
        if (!get_token(is, t)) return false;
        if (t[0] == '}') return false;
        if (t == key) {
            eat_white(is);
            char c;
            if (!is.get(c) || c != '=') return false;
            eat_blank(is);
            return true;
        }
        if (t[0] == '{') match_bracket(is);
        skip_rest_of_line(is);
    }
}

void InputGroup::SkipLine() {
    char c = '\0';
    while (c != '\n' && file_->get(c)) {
    }
    eat_white(*file_);
}

bool InputGroup::GetInt(const std::string& key, int& v, bool hasdf, int df) {
    if (!GotoToken(key) || !(*file_ >> v)) {
        if (hasdf && verbose_) std::printf("Def %s.%s = %d\n", name_.c_str(), key.c_str(), df);
        return false;
    }
    if (verbose_) std::printf("Got %s.%s = %d\n", name_.c_str(), key.c_str(), v);
    return true;
}

bool InputGroup::GetDouble(const std::string& key, double& v, bool hasdf, double df) {
    if (!GotoToken(key) || !(*file_ >> v)) {
        if (hasdf && verbose_) std::printf("Def %s.%s = %.2f\n", name_.c_str(), key.c_str(), df);
        return false;
    }
    if (verbose_) std::printf("Got %s.%s = %.2f\n", name_.c_str(), key.c_str(), v);
    return true;
}

bool InputGroup::GetString(const std::string& key, std::string& v, bool hasdf, const std::string& df) {
    if (GotoToken(key)) {
        char c;
        file_->get(c);
        if (std::isspace((unsigned char)c)) {  // "key =" with nothing after: present, empty
            if (verbose_) std::printf("%s %s.%s = %s\n", hasdf ? "Def" : "No ", name_.c_str(), key.c_str(),
                                      hasdf ? df.c_str() : "None");
            return true;
        }
        file_->putback(c);
    }
    if (!GotoToken(key) || !(*file_ >> v)) {
        if (hasdf && verbose_) std::printf("Def %s.%s = %s\n", name_.c_str(), key.c_str(), df.c_str());
        return false;
    }
    if (verbose_) std::printf("Got %s.%s = %s\n", name_.c_str(), key.c_str(), v.c_str());
    return true;
}

bool InputGroup::GetBool(const std::string& key, bool& v, bool hasdf, bool df) {
    std::string s;
    if (!GotoToken(key) || !(*file_ >> s)) {
        if (hasdf && verbose_) std::printf("Def %s.%s = %d\n", name_.c_str(), key.c_str(), (int)df);
        return false;
    }
    if (s == "true" || s == "1") v = true;
    else if (s == "false" || s == "0") v = false;
    if (verbose_) std::printf("Got %s.%s = %d\n", name_.c_str(), key.c_str(), (int)v);
    return true;
}

int InputGroup::getInt(const std::string& key) {
    int v = 0;
    if (!GetInt(key, v, false, 0)) throw InputError("there is no item: " + key);
    return v;
}
int InputGroup::getInt(const std::string& key, int def) {
    int v = 0;
    return GetInt(key, v, true, def) ? v : def;
}
double InputGroup::getDouble(const std::string& key) {
    double v = 0;
    if (!GetDouble(key, v, false, 0)) throw InputError("there is no item: " + key);
    return v;
}
double InputGroup::getDouble(const std::string& key, double def) {
    double v = 0;
    return GetDouble(key, v, true, def) ? v : def;
}
std::string InputGroup::getString(const std::string& key) {
    std::string v;
    if (!GetString(key, v, false, "")) throw InputError("there is no item: " + key);
    return v;
}
std::string InputGroup::getString(const std::string& key, const std::string& def) {
    std::string v;
    return GetString(key, v, true, def) ? v : def;
}
bool InputGroup::getBool(const std::string& key) {
    bool v = false;
    if (!GetBool(key, v, false, false)) throw InputError("there is no item: " + key);
    return v;
}
bool InputGroup::getBool(const std::string& key, bool def) {
    bool v = false;
    return GetBool(key, v, true, def) ? v : def;
}

}  // namespace dmrg
