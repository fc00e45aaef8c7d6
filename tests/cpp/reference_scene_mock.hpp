// A stand-in for the host side of betajippity/Ariel that a maintainer would bind the library
// into: the declarations of sceneCore::Scene (src/scene/scene.hpp:25-101), fluidCore::Particle
// (src/grid/macgrid.inl:36-50), geomCore::Geom / GeomInterface (src/geom/geom.hpp) and
// spaceCore::Aabb (src/spatial/aabb.hpp) that ariel::FlipSim's Scene-pointer constructor uses,
// with the same member names and signatures, and a SceneLoader with the getters main.cpp calls
// (src/main.cpp:50-54).  The behaviour is a small analytic version of the reference's: boxes
// and spheres instead of meshes, particles on the reference's sub-cell lattice
// (src/scene/scene.cpp:257-360), and an ExportParticles that records its calls.
#ifndef ARIEL_TEST_REFERENCE_SCENE_MOCK_HPP
#define ARIEL_TEST_REFERENCE_SCENE_MOCK_HPP

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace glm {
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};
}  // namespace glm

enum geomtype { SOLID = 2, FLUID = 1, AIR = 0 };

namespace spaceCore {
class Aabb {
  public:
    glm::vec3 m_min, m_max;
};
}  // namespace spaceCore

namespace geomCore {
class GeomInterface {
  public:
    virtual ~GeomInterface() {}
    virtual bool IsDynamic() = 0;
    virtual bool IsInFrame(const float& frame) = 0;
    virtual spaceCore::Aabb GetAabb(const float& frame) = 0;
    virtual bool Inside(const glm::vec3& p) = 0;  // stands in for the mesh BVH's hit counting
};

class Geom {
  public:
    GeomInterface* m_geom = nullptr;
    unsigned int m_id = 0;
};

class BoxGen : public GeomInterface {
  public:
    BoxGen(glm::vec3 lo, glm::vec3 hi) { m_box.m_min = lo; m_box.m_max = hi; }
    bool IsDynamic() override { return false; }
    bool IsInFrame(const float& frame) override { return frame == 0.0f; }
    spaceCore::Aabb GetAabb(const float&) override { return m_box; }
    bool Inside(const glm::vec3& p) override {
        return p.x > m_box.m_min.x && p.x < m_box.m_max.x && p.y > m_box.m_min.y && p.y < m_box.m_max.y &&
               p.z > m_box.m_min.z && p.z < m_box.m_max.z;
    }
    spaceCore::Aabb m_box;
};

class SphereGen : public GeomInterface {
  public:
    SphereGen(glm::vec3 c, float r) : m_c(c), m_r(r) {}
    bool IsDynamic() override { return false; }
    bool IsInFrame(const float&) override { return true; }
    spaceCore::Aabb GetAabb(const float&) override {
        spaceCore::Aabb b;
        b.m_min = glm::vec3(m_c.x - m_r, m_c.y - m_r, m_c.z - m_r);
        b.m_max = glm::vec3(m_c.x + m_r, m_c.y + m_r, m_c.z + m_r);
        return b;
    }
    bool Inside(const glm::vec3& p) override {
        float dx = p.x - m_c.x, dy = p.y - m_c.y, dz = p.z - m_c.z;
        return dx * dx + dy * dy + dz * dz < m_r * m_r;
    }
    glm::vec3 m_c;
    float m_r;
};
}  // namespace geomCore

namespace fluidCore {
struct Particle {
    glm::vec3 m_p, m_u, m_n;
    float m_density;
    float m_mass;
    int m_type;
    glm::vec3 m_t, m_t2, m_ut, m_pt;
    bool m_invalid, m_temp2, m_temp;
};
class ParticleGrid;
}  // namespace fluidCore

namespace sceneCore {
class Scene {
  public:
    ~Scene() {
        for (fluidCore::Particle* p : m_owned) delete p;
        for (geomCore::Geom* g : m_liquids) delete g->m_geom, delete g;
        for (geomCore::Geom* g : m_solids) delete g->m_geom, delete g;
    }

    // scene.cpp:257-360 on analytic geoms: sub-cell centres of each liquid AABB that are inside
    // the liquid and not inside a solid; solid particles (mass 10) inside static solids; frame 0
    // only; liquid ++ solid.
    void GenerateParticles(std::vector<fluidCore::Particle*>& particles, const glm::vec3& dimensions,
                           const float& density, fluidCore::ParticleGrid* /*pgrid*/, const int& frame) {
        if (frame != 0) return;
        const float maxd = std::max(std::max(dimensions.x, dimensions.y), dimensions.z);
        const float w = density / maxd;
        std::vector<fluidCore::Particle*> liquid, solid;
        auto lattice = [&](geomCore::GeomInterface* g, bool is_liquid, const glm::vec3& vel) {
            spaceCore::Aabb b = g->GetAabb(0.0f);
            const unsigned lo[3] = {(unsigned)(std::max(std::floor(b.m_min.x), 0.0f) / density),
                                    (unsigned)(std::max(std::floor(b.m_min.y), 0.0f) / density),
                                    (unsigned)(std::max(std::floor(b.m_min.z), 0.0f) / density)};
            const float hi[3] = {std::min(std::ceil(b.m_max.x), maxd + 1.0f) / density,
                                 std::min(std::ceil(b.m_max.y), maxd + 1.0f) / density,
                                 std::min(std::ceil(b.m_max.z), maxd + 1.0f) / density};
            for (unsigned i = lo[0]; i < hi[0]; ++i)
                for (unsigned j = lo[1]; j < hi[1]; ++j)
                    for (unsigned k = lo[2]; k < hi[2]; ++k) {
                        glm::vec3 p((i * w) + (w / 2.0f), (j * w) + (w / 2.0f), (k * w) + (w / 2.0f));
                        glm::vec3 world(p.x * maxd, p.y * maxd, p.z * maxd);
                        if (!g->Inside(world)) continue;
                        unsigned int id = 0;
                        if (is_liquid && CheckPointInsideSolidGeom(world, 0.0f, id)) continue;
                        fluidCore::Particle* q = new fluidCore::Particle();
                        q->m_p = p;
                        q->m_u = is_liquid ? vel : glm::vec3(0.0f);
                        q->m_density = 10.0f;
                        q->m_mass = is_liquid ? 1.0f : 10.0f;
                        q->m_type = is_liquid ? FLUID : SOLID;
                        q->m_invalid = false;
                        m_owned.push_back(q);
                        (is_liquid ? liquid : solid).push_back(q);
                    }
        };
        for (size_t l = 0; l < m_liquids.size(); ++l) lattice(m_liquids[l]->m_geom, true, m_liquidStartingVelocities[l]);
        for (geomCore::Geom* g : m_solids) lattice(g->m_geom, false, glm::vec3(0.0f));
        particles.clear();
        particles.insert(particles.end(), liquid.begin(), liquid.end());
        particles.insert(particles.end(), solid.begin(), solid.end());
    }

    std::vector<glm::vec3>& GetExternalForces() { return m_externalForces; }
    std::vector<geomCore::Geom*>& GetSolidGeoms() { return m_solids; }
    std::vector<geomCore::Geom*>& GetLiquidGeoms() { return m_liquids; }

    bool CheckPointInsideSolidGeom(const glm::vec3& p, const float& /*frame*/, unsigned int& solidGeomID) {
        for (size_t i = 0; i < m_solids.size(); ++i)
            if (m_solids[i]->m_geom->Inside(p)) {
                solidGeomID = (unsigned int)i;
                return true;
            }
        return false;
    }

    void ExportParticles(std::vector<fluidCore::Particle*> particles, const float& maxd, const int& frame,
                         const bool& VDB, const bool& OBJ, const bool& PARTIO) {
        ++m_exports;
        m_lastExportFrame = frame;
        m_lastExportFlags = (VDB ? 4 : 0) | (OBJ ? 2 : 0) | (PARTIO ? 1 : 0);
        m_lastExportFluid = 0;
        m_lastExportMeanY = 0.0;
        for (fluidCore::Particle* p : particles)
            if (p->m_type == FLUID && !p->m_invalid) {
                ++m_lastExportFluid;
                m_lastExportMeanY += p->m_p.y * maxd;
            }
        if (m_lastExportFluid) m_lastExportMeanY /= m_lastExportFluid;
    }

    // SceneLoader-style set-up (src/scene/sceneloader.cpp:346-443)
    void AddLiquidBox(glm::vec3 lo, glm::vec3 hi, glm::vec3 vel) {
        geomCore::Geom* g = new geomCore::Geom();
        g->m_geom = new geomCore::BoxGen(lo, hi);
        g->m_id = (unsigned int)(m_liquids.size() + m_solids.size());
        m_liquids.push_back(g);
        m_liquidStartingVelocities.push_back(vel);
    }
    void AddSolid(geomCore::GeomInterface* shape) {
        geomCore::Geom* g = new geomCore::Geom();
        g->m_geom = shape;
        g->m_id = (unsigned int)(m_liquids.size() + m_solids.size());
        m_solids.push_back(g);
    }
    void AddExternalForce(glm::vec3 force) { m_externalForces.push_back(force); }

    int m_exports = 0;
    int m_lastExportFrame = -1;
    int m_lastExportFlags = 0;
    int m_lastExportFluid = 0;
    double m_lastExportMeanY = 0.0;

  private:
    std::vector<glm::vec3> m_externalForces;
    std::vector<geomCore::Geom*> m_solids, m_liquids;
    std::vector<glm::vec3> m_liquidStartingVelocities;
    std::vector<fluidCore::Particle*> m_owned;
};

class SceneLoader {
  public:
    explicit SceneLoader(Scene* s, glm::vec3 dims, float density, float stepsize)
        : m_s(s), m_dims(dims), m_density(density), m_stepsize(stepsize) {}
    glm::vec3 GetDimensions() { return m_dims; }
    float GetDensity() { return m_density; }
    float GetStepsize() { return m_stepsize; }
    Scene* GetScene() { return m_s; }

  private:
    Scene* m_s;
    glm::vec3 m_dims;
    float m_density, m_stepsize;
};
}  // namespace sceneCore

#endif
