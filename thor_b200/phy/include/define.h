// Reference build switches and constants a module may include (src/headers/define.h); the shim
// needs none of them.
#pragma once
