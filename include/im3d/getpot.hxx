/*
 * getpot.hxx -- the parameter-file reader the segmentation class needs: the subset of
 * the GetPot format and calls that the reference uses
 * (rsfe_splitbregman_imp.hxx:582-796, examples/data).
 *
 * Format: `[section]` opens a section, `[./sub]` a subsection of the current one,
 * `[../]` closes one level; `key = value` assigns; text from the comment-start string
 * to the end of the line is ignored. A key is looked up as <prefix><key> with the
 * section names joined by '/'. A missing file behaves as an empty one (every lookup
 * returns its default), as GetPot does.
 */
#ifndef IM3D_GETPOT_HXX
#define IM3D_GETPOT_HXX

#include <cstdlib>
#include <fstream>
#include <map>
#include <string>
#include <vector>

namespace im3d
{

class getpot_file
{
    std::map<std::string, std::string> kv;
    std::string prefix;

    static std::string trim (std::string const& s)
    {
        size_t a = s.find_first_not_of (" \t\r\n");
        if (a == std::string::npos) return "";
        size_t b = s.find_last_not_of (" \t\r\n");
        return s.substr (a, b - a + 1);
    }

    std::string find (char const* key) const
    {
        auto it = kv.find (prefix + key);
        return it == kv.end() ? std::string() : it->second;
    }

public:
    explicit getpot_file (char const* filename, char const* comment_start = "#")
    {
        std::ifstream in (filename);
        std::vector<std::string> path;
        std::string line, cs = comment_start ? comment_start : "#";
        while (std::getline (in, line) )
        {
            size_t c = line.find (cs);
            if (c != std::string::npos) line = line.substr (0, c);
            line = trim (line);
            if (line.empty() ) continue;
            if (line[0] == '[')
            {
                size_t close = line.find (']');
                std::string sec = trim (line.substr (1, close == std::string::npos ? std::string::npos : close - 1) );
                if (sec == "../" || sec == "..")
                {
                    if (!path.empty() ) path.pop_back();
                }
                else if (sec.compare (0, 2, "./") == 0) path.push_back (sec.substr (2) );
                else
                {
                    path.clear();
                    path.push_back (sec);
                }
                continue;
            }
            size_t eq = line.find ('=');
            if (eq == std::string::npos) continue;
            std::string full;
            for (auto const& s : path) full += s + "/";
            kv[full + trim (line.substr (0, eq) )] = trim (line.substr (eq + 1) );
        }
    }

    void set_prefix (char const* p) { prefix = p ? p : ""; }

    int operator() (char const* key, int def) const
    {
        std::string v = find (key);
        if (v.empty() ) return def;
        char* end = nullptr;
        double d = std::strtod (v.c_str(), &end);
        return end == v.c_str() ? def : static_cast<int> (d);
    }

    double operator() (char const* key, double def) const
    {
        std::string v = find (key);
        if (v.empty() ) return def;
        char* end = nullptr;
        double d = std::strtod (v.c_str(), &end);
        return end == v.c_str() ? def : d;
    }

    std::string operator() (char const* key, char const* def) const
    {
        std::string v = find (key);
        return v.empty() ? std::string (def) : v;
    }
};

} // namespace im3d

#endif
