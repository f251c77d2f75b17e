// Stand-in for CTL's projectors/abstractprojector.h (the AbstractProjector
// interface, abstractprojector.h:65-144).  Test code only.
#ifndef CTL_STANDIN_ABSTRACTPROJECTOR_H
#define CTL_STANDIN_ABSTRACTPROJECTOR_H

#include "../ctl_standin_types.h"

namespace CTL {

class AbstractProjector : public SerializationInterface
{
public:
    virtual void configure(const AcquisitionSetup& setup) = 0;
    virtual ProjectionData project(const VolumeData& volume) = 0;
    ~AbstractProjector() override = default;
    virtual bool isLinear() const { return true; }
    QVariant toVariant() const override
    {
        QVariantMap ret = SerializationInterface::toVariant().toMap();
        ret.insert("parameters", parameter());
        return ret;
    }
    virtual QVariant parameter() const { return QVariant(); }
    virtual void setParameter(const QVariant&) {}
    virtual ProjectorNotifier* notifier() { return &_notifier; }

protected:
    AbstractProjector() = default;

private:
    ProjectorNotifier _notifier;
};

} // namespace CTL

#endif
