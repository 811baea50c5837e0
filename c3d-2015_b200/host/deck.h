// input.deck reader with the reference's format and lookup rules
// (src/input_deck_reader.cpp:17-171):
//   * one "KEY value" pair per line, '#' starts a comment;
//   * the key ends at the first space or tab, the value at the next space;
//     a third token on the line is an error;
//   * key lookup is case-insensitive, returned string values are lowercased;
//   * a bool is true only for the literal "true" (after lowercasing);
//   * numbers are parsed like atoi/atof (leading numeric prefix, 0 if none).
#pragma once
#include <string>
#include <utility>
#include <vector>

namespace c3d_host {

class InputDeck {
public:
    // Reads the file; returns false if it cannot be opened. Malformed lines are
    // reported in errors() (as the reference prints them) and skipped.
    bool read(const std::string &path);
    bool parse(const std::string &text);

    bool get(const std::string &key, std::string &value) const;
    bool get(const std::string &key, int &value) const;
    bool get(const std::string &key, double &value) const;
    bool get(const std::string &key, bool &value) const;
    bool has(const std::string &key) const;

    const std::vector<std::string> &errors() const { return errors_; }
    const std::vector<std::pair<std::string, std::string>> &entries() const { return kv_; }
    std::string print() const;

private:
    std::vector<std::pair<std::string, std::string>> kv_;
    std::vector<std::string> errors_;
};

} // namespace c3d_host
