#include "tuning.h"

#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <map>
#include <sstream>

namespace og {

const char* const ENGINE_VERSION = "b200-0.1.0";

namespace {

struct File {
    uint32_t format = 0;
    std::map<std::string, Shape> entries;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) a++;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) b--;
    return s.substr(a, b - a);
}

// A YAML scalar as written by serde: plain, or in single or double quotes.
std::string unquote(std::string s) {
    s = trim(s);
    if (s.size() >= 2 && s.front() == '"' && s.back() == '"') {
        std::string out;
        for (size_t i = 1; i + 1 < s.size(); i++) {
            if (s[i] == '\\' && i + 2 < s.size()) {
                char c = s[++i];
                out.push_back(c == 'n' ? '\n' : c == 't' ? '\t' : c);
            } else {
                out.push_back(s[i]);
            }
        }
        return out;
    }
    if (s.size() >= 2 && s.front() == '\'' && s.back() == '\'') {
        std::string out;
        for (size_t i = 1; i + 1 < s.size(); i++) {
            out.push_back(s[i]);
            if (s[i] == '\'' && i + 2 < s.size() && s[i + 1] == '\'') i++;
        }
        return out;
    }
    return s;
}

std::string quote(const std::string& s) {
    std::string out = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') out.push_back('\\');
        if (c == '\n') {
            out += "\\n";
            continue;
        }
        out.push_back(c);
    }
    return out + "\"";
}

// Splits "key: value" at the last ": " outside quotes (keys may hold ':').
bool split_kv(const std::string& line, std::string& k, std::string& v) {
    bool in_d = false, in_s = false;
    size_t at = std::string::npos;
    for (size_t i = 0; i < line.size(); i++) {
        const char c = line[i];
        if (c == '"' && !in_s) in_d = !in_d;
        else if (c == '\'' && !in_d) in_s = !in_s;
        else if (c == ':' && !in_d && !in_s && (i + 1 == line.size() || line[i + 1] == ' ')) at = i;
    }
    if (at == std::string::npos) return false;
    k = unquote(line.substr(0, at));
    v = trim(line.substr(at + 1));
    return true;
}

bool read_file(File& f) {
    const std::string path = tuning_path();
    if (path.empty()) return false;
    std::ifstream in(path);
    if (!in) return false;
    std::string line, current;
    bool in_entries = false;
    while (std::getline(in, line)) {
        if (trim(line).empty() || trim(line)[0] == '#') continue;
        size_t indent = 0;
        while (indent < line.size() && line[indent] == ' ') indent++;
        std::string k, v;
        if (!split_kv(line, k, v)) return false;
        if (indent == 0) {
            in_entries = false;
            if (k == "format") f.format = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
            else if (k == "entries") {
                in_entries = true;
                if (v == "{}") in_entries = false;
            }
        } else if (in_entries && v.empty()) {
            current = k;
            f.entries[current] = Shape{};
        } else if (in_entries && !current.empty()) {
            Shape& s = f.entries[current];
            if (k == "first") s.first = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
            else if (k == "second") s.second = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
            else if (k == "rate") s.rate = std::strtod(v.c_str(), nullptr);
            else if (k == "at") s.at = std::strtoll(v.c_str(), nullptr, 10);
            else if (k == "block") s.block = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
            else if (k == "rounds") s.rounds = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
            else if (k == "lanes_per_thread") s.lanes_per_thread = (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
        }
    }
    return true;
}

void mkdirs(const std::string& dir) {
    std::string cur;
    for (size_t i = 0; i < dir.size(); i++) {
        cur.push_back(dir[i]);
        if (dir[i] == '/' && cur.size() > 1) mkdir(cur.c_str(), 0755);
    }
    mkdir(dir.c_str(), 0755);
}

}  // namespace

std::string tuning_path() {
    if (const char* o = std::getenv("ONION_GEN_TUNING_FILE")) return o;
    std::string dir;
    if (const char* x = std::getenv("XDG_CACHE_HOME"); x && *x) dir = x;
    else if (const char* h = std::getenv("HOME"); h && *h) dir = std::string(h) + "/.cache";
    else return "";
    return dir + "/onion-gen/tuning.yaml";
}

std::string device_key(const std::string& name, const std::string& api, uint32_t threads) {
    std::string safe;
    for (char c : name) safe.push_back(c == '/' || c == '\n' ? '_' : c);
    return "device/" + safe + "/" + api + "/" + std::to_string(threads) + "/" + ENGINE_VERSION;
}

bool tuning_get(const std::string& key, Shape& out) {
    File f;
    if (!read_file(f) || f.format != 1) return false;
    auto it = f.entries.find(key);
    if (it == f.entries.end()) return false;
    out = it->second;
    return true;
}

void tuning_put(const std::string& key, const Shape& shape) {
    const std::string path = tuning_path();
    if (path.empty()) return;
    File f;
    if (!read_file(f) || f.format != 1) f = File{};
    f.format = 1;
    f.entries[key] = shape;
    std::ostringstream o;
    o << "format: 1\nentries:\n";
    for (const auto& kv : f.entries) {
        const Shape& s = kv.second;
        char rate[64];
        std::snprintf(rate, sizeof rate, "%.1f", s.rate);
        o << "  " << quote(kv.first) << ":\n"
          << "    first: " << s.first << "\n"
          << "    second: " << s.second << "\n"
          << "    rate: " << rate << "\n"
          << "    at: " << s.at << "\n";
        if (s.block) o << "    block: " << s.block << "\n";
        if (s.rounds) o << "    rounds: " << s.rounds << "\n";
        if (s.lanes_per_thread) o << "    lanes_per_thread: " << s.lanes_per_thread << "\n";
    }
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) mkdirs(path.substr(0, slash));
    // written beside and renamed, as path.with_extension("yaml.new") does
    const bool yaml = path.size() > 5 && path.compare(path.size() - 5, 5, ".yaml") == 0;
    const std::string tmp = yaml ? path.substr(0, path.size() - 5) + ".yaml.new" : path + ".new";
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return;
        out << o.str();
        if (!out) return;
    }
    std::rename(tmp.c_str(), path.c_str());
}

int64_t unix_now() { return (int64_t)std::time(nullptr); }

}  // namespace og
