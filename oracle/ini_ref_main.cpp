// Test-only checker: a command-line driver around the reference's own
// IniConfig (modules/litho-io/src/io/ini_config.cpp, compiled unmodified from
// the reference tree into oracle/_ref/ini_ref by oracle/Makefile).  The INI
// tests send it the same queries they send lithoinv3d_b200.config.IniConfig
// and compare the answers.
//
//   ini_ref <file.ini>            then one query per stdin line, fields
//                                 separated by tabs:
//     S <section> <key> <default>  getString
//     D <section> <key> <default>  getDouble (default parsed with strtod)
//     I <section> <key> <default>  getInt
//     B <section> <key> <0|1>      getBool
//     H <section>                  hasSection
//     L                            sections(), tab-separated
//     W <path>                     save(path)
// One answer line per query: doubles as %.17g, bools as 0 / 1.
#include <litho_invert/io/ini_config.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

static std::vector<std::string> split_tabs(const std::string& s) {
    std::vector<std::string> out;
    size_t b = 0;
    for (;;) {
        size_t e = s.find('\t', b);
        out.push_back(s.substr(b, e == std::string::npos ? std::string::npos : e - b));
        if (e == std::string::npos) break;
        b = e + 1;
    }
    return out;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ini_ref <file.ini>\n");
        return 2;
    }
    litho_invert::IniConfig ini;
    std::printf("%d\n", ini.load(argv[1]) ? 1 : 0);
    std::string line;
    while (std::getline(std::cin, line)) {
        std::vector<std::string> f = split_tabs(line);
        const std::string& op = f[0];
        if (op == "S" && f.size() == 4) {
            std::printf("%s\n", ini.getString(f[1], f[2], f[3]).c_str());
        } else if (op == "D" && f.size() == 4) {
            std::printf("%.17g\n", ini.getDouble(f[1], f[2], std::strtod(f[3].c_str(), nullptr)));
        } else if (op == "I" && f.size() == 4) {
            std::printf("%d\n", ini.getInt(f[1], f[2], std::atoi(f[3].c_str())));
        } else if (op == "B" && f.size() == 4) {
            std::printf("%d\n", ini.getBool(f[1], f[2], f[3] == "1") ? 1 : 0);
        } else if (op == "H" && f.size() == 2) {
            std::printf("%d\n", ini.hasSection(f[1]) ? 1 : 0);
        } else if (op == "L") {
            std::vector<std::string> s = ini.sections();
            for (size_t i = 0; i < s.size(); ++i) std::printf(i ? "\t%s" : "%s", s[i].c_str());
            std::printf("\n");
        } else if (op == "W" && f.size() == 2) {
            ini.save(f[1]);
            std::printf("saved\n");
        } else {
            std::printf("?\n");
        }
        std::fflush(stdout);
    }
    return 0;
}
