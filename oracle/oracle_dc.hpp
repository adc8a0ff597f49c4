// CPU oracle dual-contouring mesher (TEST INFRASTRUCTURE ONLY).
#pragma once
