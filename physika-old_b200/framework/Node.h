// Node.h -- Base / Module / Node / SceneGraph subset (Framework/Framework/Base.h,
// Module.h:18-105, ModuleCompute.h:6-19, ModuleConstraint.h:8-28,
// NumericalIntegrator.h:6-35, NumericalModel.h:7-22, Node.h:36-375,
// SceneGraph.h:9-107).
#pragma once
#include <list>
#include <map>

#include "Framework.h"

namespace PhysIKA {

class Node;

class Base {
public:
    virtual ~Base() = default;
};

class Module : public Base {
public:
    explicit Module(std::string name = "default") : m_module_name(std::move(name)) {}
    ~Module() override = default;

    // Module::initialize (Module.cpp:22-31): runs initializeImpl once.
    bool initialize()
    {
        if (m_initialized) return true;
        m_initialized = initializeImpl();
        return m_initialized;
    }
    virtual void begin() {}
    virtual bool execute() { return true; }
    virtual void end() {}
    void setName(std::string name) { m_module_name = std::move(name); }
    std::string getName() const { return m_module_name; }
    void setParent(Node* node) { m_node = node; }
    Node* getParent()
    {
        if (m_node == nullptr) Log::sendMessage(Log::Error, "Parent node is not set!");
        return m_node;
    }
    bool isInitialized() const { return m_initialized; }
    virtual std::string getModuleType() { return "Module"; }

protected:
    virtual bool initializeImpl() { return true; }

private:
    Node* m_node = nullptr;
    std::string m_module_name;
    bool m_initialized = false;
};

class ComputeModule : public Module {
public:
    bool execute() override
    {
        compute();
        return true;
    }
    virtual void compute() {}
    std::string getModuleType() override { return "ComputeModule"; }
};

class ConstraintModule : public Module {
public:
    bool execute() override { return constrain(); }
    virtual bool constrain() { return true; }
    std::string getModuleType() override { return "ConstraintModule"; }
};

class NumericalIntegrator : public Module {
public:
    virtual void begin() override {}
    virtual void end() override {}
    virtual bool integrate() { return true; }
    std::string getModuleType() override { return "NumericalIntegrator"; }
};

class NumericalModel : public Module {
public:
    virtual void step(float dt) { (void)dt; }
    std::string getModuleType() override { return "NumericalModel"; }
};

// SceneGraph singleton: gravity and scene bounds (SceneGraph.h:57-80).
class SceneGraph {
public:
    static SceneGraph& getInstance()
    {
        static SceneGraph g;
        return g;
    }
    Vector3f getGravity() const { return m_gravity; }
    void setGravity(Vector3f g) { m_gravity = g; }
    Vector3f getLowerBound() const { return m_lower; }
    Vector3f getUpperBound() const { return m_upper; }
    void setLowerBound(Vector3f v) { m_lower = v; }
    void setUpperBound(Vector3f v) { m_upper = v; }

private:
    Vector3f m_gravity{0.0f, -9.8f, 0.0f};
    Vector3f m_lower{0.0f, 0.0f, 0.0f};
    Vector3f m_upper{1.0f, 1.0f, 1.0f};
};

// Node: owns modules; dt (Node.h:72, default 0.001 Node.cpp:15).
class Node : public Base {
public:
    explicit Node(std::string name = "default") : m_name(std::move(name)) {}
    ~Node() override = default;

    float getDt() const { return m_dt; }
    void setDt(float dt) { m_dt = dt; }
    std::string getName() const { return m_name; }

    template <class TModule>
    std::shared_ptr<TModule> addComputeModule(std::string name)
    {
        auto m = std::make_shared<TModule>();
        m->setName(name);
        m->setParent(this);
        m_compute.push_back(m);
        m_modules[name] = m;
        return m;
    }
    template <class TModule>
    std::shared_ptr<TModule> addConstraintModule(std::string name)
    {
        auto m = std::make_shared<TModule>();
        m->setName(name);
        return std::dynamic_pointer_cast<TModule>(addConstraintModule(m));
    }
    std::shared_ptr<ConstraintModule> addConstraintModule(std::shared_ptr<ConstraintModule> m)
    {
        m->setParent(this);
        m_constraints.push_back(m);
        m_modules[m->getName()] = m;
        return m;
    }
    template <class TModule>
    std::shared_ptr<TModule> setNumericalIntegrator(std::string name)
    {
        auto m = std::make_shared<TModule>();
        m->setName(name);
        m->setParent(this);
        m_integrator = m;
        m_modules[name] = m;
        return m;
    }
    template <class TModule>
    std::shared_ptr<TModule> setNumericalModel(std::string name)
    {
        auto m = std::make_shared<TModule>();
        m->setName(name);
        m->setParent(this);
        m_model = m;
        m_modules[name] = m;
        return m;
    }
    template <class TModule>
    std::shared_ptr<TModule> getModule(std::string name)
    {
        auto it = m_modules.find(name);
        return it == m_modules.end() ? nullptr : std::dynamic_pointer_cast<TModule>(it->second);
    }
    bool deleteModule(std::shared_ptr<Module> m)
    {
        m_modules.erase(m->getName());
        m_constraints.remove_if([&](const std::shared_ptr<ConstraintModule>& c) { return c == m; });
        m_compute.remove_if([&](const std::shared_ptr<ComputeModule>& c) { return c == m; });
        return true;
    }
    std::shared_ptr<NumericalModel> getNumericalModel() { return m_model; }
    std::shared_ptr<NumericalIntegrator> getNumericalIntegrator() { return m_integrator; }

    // Node::initialize / advance (Node.cpp:96-169): the model steps the node.
    virtual bool initialize() { return m_model ? m_model->initialize() : true; }
    virtual void advance(float dt)
    {
        if (m_model) m_model->step(dt);
    }

protected:
    std::string m_name;
    float m_dt = 0.001f;
    std::shared_ptr<NumericalModel> m_model;
    std::shared_ptr<NumericalIntegrator> m_integrator;
    std::list<std::shared_ptr<ComputeModule>> m_compute;
    std::list<std::shared_ptr<ConstraintModule>> m_constraints;
    std::map<std::string, std::shared_ptr<Module>> m_modules;
};

}  // namespace PhysIKA
