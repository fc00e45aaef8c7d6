// TEST INFRASTRUCTURE ONLY: force-included after prelude.hpp when oracle/ref_mesh_driver.cpp
// compiles betajippity/Ariel's mesh sources (src/spatial/aabb.cpp, src/geom/obj/obj.cpp) into
// oracle/_ref/.  utilities.h is kept out by prelude.hpp; this declares in its place the
// utilityCore helpers those two files call (OBJ parsing and matrix transforms, neither of which
// the pinned ray-triangle test reaches) and the REALLY_BIG_NUMBER constant of utilities.h.
#ifndef ARIEL_REFSHIM_MESH_PRELUDE_HPP
#define ARIEL_REFSHIM_MESH_PRELUDE_HPP

#include <string>
#include <vector>

#define REALLY_BIG_NUMBER 1000000000000000000

namespace utilityCore {
// split at any character of `separator`, dropping empty tokens
inline std::vector<std::string> tokenizeString(std::string str, std::string separator) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : str) {
        if (separator.find(ch) != std::string::npos) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += ch;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}
inline std::string getFirstNCharactersOfString(std::string s, int n) {
    return s.substr(0, (size_t)(n < 0 ? 0 : n));
}
// column-major matrix times vector
inline glm::vec4 multiply(glm::mat4 m, glm::vec4 v) {
    glm::vec4 r;
    r.x = m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z + m.c[3].x * v.w;
    r.y = m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z + m.c[3].y * v.w;
    r.z = m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z + m.c[3].z * v.w;
    r.w = m.c[0].w * v.x + m.c[1].w * v.y + m.c[2].w * v.z + m.c[3].w * v.w;
    return r;
}
}  // namespace utilityCore

#endif
