// Stand-in for the reference's engine/gui/GUISettings.h (which pulls in ImGui through
// GUIElements.h) when its CUDA path tracer is compiled on its own for timing on the
// device. Test infrastructure only. It gives the settings structs of
// application/CUDAPathTracer/GUI/PathTracingSettings.h the value types they use — a
// labelled value with a range that reads as the value — and no drawing.
#pragma once
#include <string>
#include <vector>

struct GUIElement
{
    explicit GUIElement(const std::string& label) : label(label) {}
    virtual ~GUIElement() {}
    std::string label;
};

template <class T>
struct Slider : GUIElement
{
    Slider(const std::string& label, T value, T min, T max) : GUIElement(label), value(value), min(min), max(max) {}
    operator T() const { return value; }
    T value, min, max;
};

struct SliderFloat : Slider<float>
{
    SliderFloat(const std::string& label, float value, float min, float max) : Slider(label, value, min, max) {}
};

struct SliderInt : Slider<int>
{
    SliderInt(const std::string& label, int value, int min, int max) : Slider(label, value, min, max) {}
};

struct CheckBox : GUIElement
{
    CheckBox(const std::string& label, bool value) : GUIElement(label), value(value) {}
    operator bool() const { return value; }
    bool value;
};

struct GUISettings
{
    std::vector<GUIElement*> guiElements;
};
