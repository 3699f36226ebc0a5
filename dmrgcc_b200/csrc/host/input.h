// Input-file reader with the reference's format and semantics
// (InputGroup, src/util/input.{h,cc}): brace groups "name { key = value ... }",
// nested groups, tokens of letters/underscore/digits, one key per line, a
// table read with >> after SkipLine().  get*(key) without a default fails when
// the key is missing (the reference exits; here an InputError is thrown);
// get*(key, default) falls back.  Lookups print "Got"/"Def" lines like the
// reference when verbose.
#pragma once

#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>

namespace dmrg {

struct InputError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class InputGroup {
public:
    InputGroup(const std::string& file_name, const std::string& group_name, bool verbose = true);
    InputGroup(InputGroup& parent, const std::string& name);

    const std::string& name() const { return name_; }
    std::ifstream& file() { return *file_; }

    bool GotoGroup();
    bool GotoToken(const std::string& key);
    void SkipLine();

    int getInt(const std::string& key);
    int getInt(const std::string& key, int def);
    double getDouble(const std::string& key);
    double getDouble(const std::string& key, double def);
    std::string getString(const std::string& key);
    std::string getString(const std::string& key, const std::string& def);
    bool getBool(const std::string& key);
    bool getBool(const std::string& key, bool def);

private:
    bool GetInt(const std::string& key, int& v, bool hasdf, int df);
    bool GetDouble(const std::string& key, double& v, bool hasdf, double df);
    bool GetString(const std::string& key, std::string& v, bool hasdf, const std::string& df);
    bool GetBool(const std::string& key, bool& v, bool hasdf, bool df);
    void reopen();

    std::string file_name_;
    std::shared_ptr<std::ifstream> file_;
    InputGroup* parent_ = nullptr;
    std::string name_;
    bool verbose_ = true;
};

}  // namespace dmrg
