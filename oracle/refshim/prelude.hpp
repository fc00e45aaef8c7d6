// TEST INFRASTRUCTURE ONLY: force-included (`g++ -include`) ahead of betajippity/Ariel's own FLIP
// sources when oracle/ref_driver.cpp compiles them into oracle/_ref/.  It stands in for the
// headers of that path which need libraries absent here, by defining their include guards
// first and declaring in their place only what the FLIP step calls:
//
//  * UTILITIES_H (src/utilities/utilities.h): the Takua string/matrix helpers.  The FLIP step
//    uses none of them; only the HOST/DEVICE macros and the glm include are kept.
//  * RAY_HPP (src/ray/ray.hpp): rayCore::Ray and rayCore::Intersection with the fields the
//    step reads, the default contents that src/ray/ray.cpp:15-17 and :56-58 give them,
//    Intersection::CompareClosestAgainst as src/ray/ray.cpp:83-98 defines it, and (for the
//    mesh sources) Ray::GetPointAlongRay and the full Intersection constructor of ray.cpp.
//  * LEVELSET_HPP (src/grid/levelset.hpp): the OpenVDB level set.  Only
//    ProjectPointsToSurface and GetCell are called by the step; the driver implements them on
//    analytic spheres.
//  * SCENE_HPP (src/scene/scene.hpp): sceneCore::Scene with the member functions the step calls
//    (src/scene/scene.hpp:31-62); the driver implements them on analytic spheres and on a
//    particle list handed over by the test (the reference's JSON scenes, meshes and Partio
//    export are not on the path).
#ifndef ARIEL_REFSHIM_PRELUDE_HPP
#define ARIEL_REFSHIM_PRELUDE_HPP

// Every standard header the reference's sources use, included before any of them so that the
// driver's `#define private public` (test access to FlipSim's stages) never reaches one.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <istream>
#include <iterator>
#include <ostream>
#include <sstream>
#include <string>
#include <vector>

#include <glm/glm.hpp>
#include <tbb/tbb.h>

#define UTILITIES_H
#define HOST
#define DEVICE

#define RAY_HPP
namespace rayCore {
class Ray {
  public:
    Ray() : m_origin(0.0f), m_direction(0.0f, 1.0f, 0.0f), m_trackingID(0), m_frame(0.0f) {}
    // src/ray/ray.cpp:40-42
    glm::vec3 GetPointAlongRay(const float& distance) const { return m_origin + distance * m_direction; }
    glm::vec3 m_origin;
    glm::vec3 m_direction;
    unsigned int m_trackingID;
    float m_frame;
};

class Intersection {
  public:
    Intersection()
        : m_point(0.0f), m_normal(1.0f, 0.0f, 0.0f), m_uv(0.0f), m_objectID(0), m_primID(0), m_hit(false) {}
    Intersection(bool hit, const glm::vec3& point, const glm::vec3& normal)
        : m_point(point), m_normal(normal), m_uv(0.0f), m_objectID(0), m_primID(0), m_hit(hit) {}
    // src/ray/ray.cpp:60-64
    Intersection(const bool& hit, const glm::vec3& point, const glm::vec3& normal, const glm::vec2& uv,
                 const unsigned int& objectID, const unsigned int& primID)
        : m_point(point), m_normal(normal), m_uv(uv), m_objectID(objectID), m_primID(primID), m_hit(hit) {}
    Intersection CompareClosestAgainst(const Intersection& b, const glm::vec3& point) const {
        if (m_hit && !b.m_hit) return *this;
        if (!m_hit && b.m_hit) return b;
        float distanceA = glm::length(m_point - point);
        float distanceB = glm::length(b.m_point - point);
        return distanceA <= distanceB ? *this : b;
    }
    glm::vec3 m_point;
    glm::vec3 m_normal;
    glm::vec2 m_uv;
    unsigned int m_objectID;
    unsigned int m_primID;
    bool m_hit;
};
}  // namespace rayCore

namespace sceneCore {
class Scene;
}  // namespace sceneCore

namespace fluidCore {
struct Particle;
class ParticleGrid;
}  // namespace fluidCore

#define LEVELSET_HPP
namespace fluidCore {
class LevelSet {
  public:
    void ProjectPointsToSurface(std::vector<Particle*>& particles, const float& pscale);
    float GetCell(const int& x, const int& y, const int& z);
    sceneCore::Scene* m_owner = nullptr;
};
}  // namespace fluidCore

#define SCENE_HPP
namespace sceneCore {
class Scene {
  public:
    void GenerateParticles(std::vector<fluidCore::Particle*>& particles, const glm::vec3& dimensions,
                           const float& density, fluidCore::ParticleGrid* pgrid, const int& frame);
    std::vector<glm::vec3>& GetExternalForces();
    fluidCore::LevelSet* GetSolidLevelSet();
    fluidCore::LevelSet* GetLiquidLevelSet();
    void BuildSolidGeomLevelSet(const int& frame);
    void BuildPermaSolidGeomLevelSet();
    void ExportParticles(std::vector<fluidCore::Particle*> particles, const float& maxd, const int& frame,
                         const bool& VDB, const bool& OBJ, const bool& PARTIO);
    rayCore::Intersection IntersectSolidGeoms(const rayCore::Ray& r);
    bool CheckPointInsideSolidGeom(const glm::vec3& p, const float& frame, unsigned int& solidGeomID);

    // analytic solid spheres in world (grid) units, and the frame-0 particle list
    std::vector<glm::vec3> m_sphereCenters;
    std::vector<float> m_sphereRadii;
    std::vector<glm::vec3> m_externalForces;
    std::vector<fluidCore::Particle*> m_initialParticles;
    fluidCore::LevelSet m_solidLevelSet;
    fluidCore::LevelSet m_liquidLevelSet;
};
}  // namespace sceneCore

#endif
