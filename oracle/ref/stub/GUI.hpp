// Stand-in for the reference's core/GUI.hpp (OpenGL / ImGui viewer), which
// dataGen.cu includes but whose sampling functions do not use: lets the
// reference's dataGen.cu compile for the test harness without a GUI stack.
#pragma once
