// parameters.txt and raw float32 file handling, compatible with the reference's
// file_manager (src/utils/file_manager/file_manager.cpp) including its quirks, so that the
// reference's parameter files and data layouts are this library's API unchanged:
//  * the first line that STARTS with the key wins (a prefix match);
//  * the value starts two characters after '=' and ends at '#';
//  * lines starting with '#' or ' ' are skipped;
//  * a value starting with '"' (or '[') has those characters removed WITHOUT shrinking the
//    string (std::remove, no erase), so a quoted value keeps trailing leftovers unless
//    it was followed by at least two spaces or a comment -- then all spaces are erased.
#include <algorithm>
#include <cctype>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "tomo_b200_interface.hpp"

bool str2bool(std::string s)
{
    for (char &c : s) c = (char)std::tolower((unsigned char)c);
    bool b = false;
    std::istringstream(s) >> std::boolalpha >> b;
    return b;
}

void read_binary_float(std::string path, float *array, int n)
{
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f.is_open()) throw std::invalid_argument("Error: file could not be opened!");
    f.read(reinterpret_cast<char *>(array), (std::streamsize)n * (std::streamsize)sizeof(float));
}

void write_binary_float(std::string path, float *array, int n)
{
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f.is_open()) throw std::invalid_argument("Error: file could not be opened!");
    f.write(reinterpret_cast<const char *>(array), (std::streamsize)n * (std::streamsize)sizeof(float));
    std::cout << "Binary file " + path + " was succesfully written." << std::endl;
}

void read_text_file(std::string path, std::vector<std::string> &elements)
{
    std::ifstream f(path, std::ios::in);
    if (!f.is_open()) throw std::invalid_argument("Error: file could not be opened!");
    std::string line;
    while (std::getline(f, line)) elements.push_back(line);
}

std::string catch_parameter(std::string target, std::string file)
{
    std::string value;
    std::ifstream in(file);
    if (in.is_open()) {
        std::string line;
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#' || line[0] == ' ') continue;
            if (line.compare(0, target.size(), target) != 0) continue;
            // two characters after '=' (an absent '=' wraps to index 1, as the reference's
            // int arithmetic on std::string::npos does)
            const int start = (int)(line.find('=') + 2);
            for (int i = start; i < (int)line.size(); i++) {
                if (line[(size_t)i] == '#') break;
                value += line[(size_t)i];
            }
            break;
        }
    }
    if (value.find('"') == 0) {
        (void)std::remove(value.begin(), value.end(), '"');
    } else if (value.find('[') == 0) {
        (void)std::remove(value.begin(), value.end(), '[');
        (void)std::remove(value.begin(), value.end(), ']');
    }
    value.erase(std::remove(value.begin(), value.end(), ' '), value.end());
    return value;
}

std::vector<std::string> split(std::string s, char delimiter)
{
    std::vector<std::string> out;
    std::istringstream in(s);
    std::string tok;
    while (std::getline(in, tok, delimiter)) out.push_back(tok);
    return out;
}

// trilinear (src/utils/interpolation/trilinear.cpp:3-20): same weights and order.
float trilinear(float c000, float c001, float c100, float c101, float c010, float c011, float c110, float c111,
                float x0, float x1, float y0, float y1, float z0, float z1, float x, float y, float z)
{
    const float tx = (x - x0) / (x1 - x0), ty = (y - y0) / (y1 - y0), tz = (z - z0) / (z1 - z0);
    const float a0 = c000 * (1 - tx) + c100 * tx;
    const float a1 = c001 * (1 - tx) + c101 * tx;
    const float b0 = c010 * (1 - tx) + c110 * tx;
    const float b1 = c011 * (1 - tx) + c111 * tx;
    const float e0 = a0 * (1 - ty) + b0 * ty;
    const float e1 = a1 * (1 - ty) + b1 * ty;
    return e0 * (1 - tz) + e1 * tz;
}
