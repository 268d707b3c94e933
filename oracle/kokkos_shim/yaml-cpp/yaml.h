/* Stand-in for yaml-cpp in the reference build (test infrastructure only): the reference
 * headers compiled here only declare functions taking a YAML::Node, whose definitions
 * (configuration/*.cpp) are not part of the build. */
#pragma once
namespace YAML {
class Node;
}
