// Test-infrastructure shim: the reference's OBJ loader wraps tinyobjloader,
// which is not installed. The SPH hot path never loads meshes; the symbol is
// only referenced from scene construction and test bodies.
#include "scene/loader.h"
#include <stdexcept>

Mesh load_mesh_from_obj(const std::filesystem::path&,
    const std::vector<std::string>, const std::optional<std::string>)
{
    throw std::runtime_error("OBJ loading is not available in the oracle build");
}
