#include "deck.h"

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace c3d_host {

static std::string lower(std::string s)
{
    for (char &c : s)
        c = (char)std::tolower((unsigned char)c);
    return s;
}

bool InputDeck::read(const std::string &path)
{
    std::ifstream f(path);
    if (!f)
        return false;
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str());
}

bool InputDeck::parse(const std::string &text)
{
    std::istringstream in(text);
    std::string line;
    int lineNumber = 0;
    while (std::getline(in, line)) {
        ++lineNumber;
        size_t hash = line.find('#');
        if (hash != std::string::npos)
            line.resize(hash);
        if (!line.empty() && line.back() == '\r')
            line.pop_back();
        // key: first token delimited by spaces or tabs
        size_t p = line.find_first_not_of(" \t");
        if (p == std::string::npos)
            continue;
        size_t e = line.find_first_of(" \t", p);
        std::string key = line.substr(p, e == std::string::npos ? std::string::npos : e - p);
        // value: next token delimited by spaces only
        std::string value;
        bool haveValue = false, extra = false;
        if (e != std::string::npos) {
            size_t rest = e + 1;
            size_t v0 = line.find_first_not_of(' ', rest);
            if (v0 != std::string::npos) {
                size_t v1 = line.find(' ', v0);
                value = line.substr(v0, v1 == std::string::npos ? std::string::npos : v1 - v0);
                haveValue = true;
                if (v1 != std::string::npos && line.find_first_not_of(' ', v1) != std::string::npos)
                    extra = true;
            }
        }
        if (!haveValue)
            errors_.push_back("Error in input file at line: " + std::to_string(lineNumber));
        if (extra) {
            errors_.push_back("Error in input file at line: " + std::to_string(lineNumber));
            continue;
        }
        kv_.emplace_back(key, value);
    }
    return true;
}

bool InputDeck::get(const std::string &key, std::string &value) const
{
    std::string k = lower(key);
    for (const auto &kv : kv_) {
        if (lower(kv.first) == k) {
            value = lower(kv.second);
            return true;
        }
    }
    return false;
}

bool InputDeck::has(const std::string &key) const
{
    std::string v;
    return get(key, v);
}

bool InputDeck::get(const std::string &key, int &value) const
{
    std::string s;
    if (!get(key, s))
        return false;
    value = std::atoi(s.c_str());
    return true;
}

bool InputDeck::get(const std::string &key, double &value) const
{
    std::string s;
    if (!get(key, s))
        return false;
    value = std::atof(s.c_str());
    return true;
}

bool InputDeck::get(const std::string &key, bool &value) const
{
    std::string s;
    if (!get(key, s))
        return false;
    value = (s == "true");
    return true;
}

std::string InputDeck::print() const
{
    std::string out = "--- Input Deck ---\n";
    for (const auto &kv : kv_)
        out += kv.first + " = " + kv.second + "\n";
    return out;
}

} // namespace c3d_host
