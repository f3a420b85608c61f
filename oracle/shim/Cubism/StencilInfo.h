// Oracle test infrastructure: Cubism's StencilInfo header is included by the
// reference (Definitions.h:28) but none of its symbols are used on this path.
#pragma once
namespace cubism { struct StencilInfo {}; }
