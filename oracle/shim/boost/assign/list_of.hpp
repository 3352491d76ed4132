// Empty stand-in: the reference includes this header in its Gmsh element table file
// without using it.
#pragma once
