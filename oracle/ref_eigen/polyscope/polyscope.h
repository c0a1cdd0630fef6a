// Stand-in for the Polyscope viewer API that the reference's CPU sources name in their
// visualisation functions (Cell::visualize, the hermite_update debug views, contouring's
// viewer hooks), so those files compile without a graphics stack. TEST INFRASTRUCTURE ONLY:
// the dual-contouring path the tests drive never calls them; every call here does nothing.
#pragma once
#include <string>

namespace polyscope {

enum class PointRenderMode { Sphere = 0, Quad = 1 };

// One object for every structure and quantity: each setter accepts anything and returns the
// object, so chained calls compile.
struct Handle {
    template <typename... A> Handle* setPointColor(A&&...) { return this; }
    template <typename... A> Handle* setPointRadius(A&&...) { return this; }
    template <typename... A> Handle* setEnabled(A&&...) { return this; }
    template <typename... A> Handle* addColorQuantity(A&&...) { return this; }
    template <typename... A> Handle* addVectorQuantity(A&&...) { return this; }
    template <typename... A> Handle* addScalarQuantity(A&&...) { return this; }
    template <typename... A> Handle* setVectorColor(A&&...) { return this; }
    template <typename... A> Handle* setRadius(A&&...) { return this; }
    template <typename... A> Handle* setPointRenderMode(A&&...) { return this; }
    template <typename... A> Handle* setColor(A&&...) { return this; }
    template <typename... A> Handle* setTransparency(A&&...) { return this; }
    template <typename... A> Handle* setSurfaceColor(A&&...) { return this; }
    template <typename... A> Handle* setPointRadiusQuantity(A&&...) { return this; }
    template <typename... A> Handle* setMapRange(A&&...) { return this; }
    template <typename... A> Handle* setEdgeWidth(A&&...) { return this; }
    template <typename... A> Handle* setEdgeColor(A&&...) { return this; }
    template <typename... A> Handle* setVectorLengthScale(A&&...) { return this; }
    template <typename... A> Handle* setVectorRadius(A&&...) { return this; }
    template <typename... A> Handle* setSmoothShade(A&&...) { return this; }
    template <typename... A> Handle* updatePointPositions(A&&...) { return this; }
    template <typename... A> Handle* updateVertexPositions(A&&...) { return this; }
    size_t nPoints() const { return 0; }
};
using PointCloud = Handle;
using SurfaceMesh = Handle;
using CurveNetwork = Handle;

inline Handle* handle() {
    static Handle h;
    return &h;
}
template <typename... A> inline Handle* registerPointCloud(A&&...) { return handle(); }
template <typename... A> inline Handle* registerSurfaceMesh(A&&...) { return handle(); }
template <typename... A> inline Handle* registerCurveNetwork(A&&...) { return handle(); }
template <typename... A> inline Handle* getPointCloud(A&&...) { return handle(); }
template <typename... A> inline Handle* getSurfaceMesh(A&&...) { return handle(); }
template <typename... A> inline void removeStructure(A&&...) {}
template <typename... A> inline void removeAllStructures(A&&...) {}
template <typename... A> inline void init(A&&...) {}
template <typename... A> inline void show(A&&...) {}
template <typename... A> inline bool hasPointCloud(A&&...) { return false; }

}  // namespace polyscope
